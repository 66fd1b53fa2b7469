// scft_main.cpp -- drop-in driver `scft_b200 [input.dat]` for the reference
// program (scft.cu:869-1191): same input.dat keys, win<ii> field files,
// rhoA_<ii>.vtk / rhocB_<ii>.vtk dumps, FEs and check files and progress
// lines, on one B200 through the C ABI.  Every replica lives on the GPU; there
// is no MPI.
//
// Extra input.dat keys (unknown keys are ignored, as in the reference):
//   strn      replicas on the string (compile-time 48 in the reference, scft.cu:35)
//   nsterp    solve_field iterations (4000 in the reference, scft.cu:1102)
//   precision 64 (default, the reference arithmetic) or 32 (FP32 propagator bulk)
//   batched   1 (default): replicas advance together; 0: one at a time
//   errtol    stop when errtot <= errtol (0 = never, as the reference)
//   handover  with precision 32: when errtot <= handover, or after 200
//             iterations without 1 % progress, the fields move to an FP64
//             context and the same run continues there (0 = never); the FP32
//             propagator's error floor then no longer limits errtol or F
//   checkpoint 1: also write the binary FP64 checkpoint `fields.ckpt` wherever
//             the win files are written
//   restart   1: start from `fields.ckpt` (box and fields) instead of win files
//   fcont     1: continuous A fraction (no rounding of f; junction step inside
//             the chain), 0 (default): the reference's rounded f
// Environment: SCFT_DRY_RUN=1 prints the resolved input and the start fields
// and exits before any device call.
#include <csignal>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <algorithm>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <thread>
#include <vector>

#include "../../include/scft_b200.h"

namespace {

volatile std::sig_atomic_t g_sig = 0;
time_t g_time0;

void on_sigint(int) { g_sig = 7; }  // scft.cu:299-302

std::string tistr()  // scft.cu:322-345
{
    long tisec = (long)(time(nullptr) - g_time0);
    const int lm = 60, lh = 60 * lm, ld = 24 * lh;
    int days = tisec / ld, hours = (tisec - days * ld) / lh, mins = (tisec - days * ld - hours * lh) / lm;
    int secs = tisec - days * ld - hours * lh - mins * lm;
    char b[64];
    if (days > 0)
        snprintf(b, sizeof b, "%d, %02d:%02d:%02d", days, hours, mins, secs);
    else if (hours > 0)
        snprintf(b, sizeof b, "%d:%02d:%02d", hours, mins, secs);
    else if (mins > 0)
        snprintf(b, sizeof b, "%d:%02d", mins, secs);
    else
        snprintf(b, sizeof b, "%ds", secs);
    return b;
}

// `key = v1 v2 ...`, '#' comments, whitespace-stripped keys (scft.cu:80-114)
std::unordered_map<std::string, std::vector<double>> read_parameters(const std::string &fn)
{
    std::unordered_map<std::string, std::vector<double>> params;
    std::ifstream file(fn);
    std::string line;
    while (std::getline(file, line)) {
        size_t c = line.find('#');
        if (c != std::string::npos) line.erase(c);
        auto notsp = [](unsigned char ch) { return !std::isspace(ch); };
        line.erase(line.begin(), std::find_if(line.begin(), line.end(), notsp));
        line.erase(std::find_if(line.rbegin(), line.rend(), notsp).base(), line.end());
        if (line.empty()) continue;
        std::istringstream iss(line);
        std::string key;
        if (std::getline(iss, key, '=')) {
            key.erase(std::remove_if(key.begin(), key.end(), ::isspace), key.end());
            std::vector<double> v;
            double x;
            while (iss >> x) v.push_back(x);
            params[key] = v;
        }
    }
    return params;
}

int count_lines(const std::string &fn)  // lines(), scft.cu:259-280
{
    FILE *fp = fopen(fn.c_str(), "r");
    if (!fp) {
        std::cerr << "Failed to open file: " << fn << std::endl;
        return -1;
    }
    int n = 0, ch;
    while ((ch = fgetc(fp)) != EOF)
        if (ch == '\n') n++;
    fclose(fp);
    return n;
}

bool fexist(const std::string &fn)
{
    FILE *f = fopen(fn.c_str(), "r");
    if (!f) return false;
    fclose(f);
    return true;
}

// Formats rows [0, nrows) with fmt_row(row, std::string &out) (appending), in
// parallel chunks of rows, and writes the chunks in order: the bytes are those
// of the one-fprintf-per-value loops of the reference, produced by several
// threads (the ASCII files of a 128^3 string run to hundreds of MB).
template <class Fmt>
void write_rows(FILE *out, long nrows, Fmt fmt_row)
{
    const long nthr = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const long chunk = std::max(1L, std::min(65536L, (nrows + nthr - 1) / nthr));
    const long nchunks = (nrows + chunk - 1) / chunk;
    for (long c0 = 0; c0 < nchunks; c0 += nthr) {
        const long c1 = std::min(nchunks, c0 + nthr);
        std::vector<std::string> bufs(c1 - c0);
        std::vector<std::thread> th;
        for (long c = c0; c < c1; c++)
            th.emplace_back([&, c]() {
                std::string &b = bufs[c - c0];
                const long r0 = c * chunk, r1 = std::min(nrows, r0 + chunk);
                for (long r = r0; r < r1; r++) fmt_row(r, b);
            });
        for (auto &t : th) t.join();
        for (auto &b : bufs) fwrite(b.data(), 1, b.size(), out);
    }
}

// appends printf(fmt, v) (a %lf conversion prints at most 317 characters)
inline void append_f(std::string &o, const char *fmt, double v)
{
    char t[400];
    const int n = snprintf(t, sizeof t, fmt, v);
    o.append(t, (size_t)std::min(std::max(n, 0), (int)sizeof t - 1));
}

void tovtk(const std::string &fname, const int *m, const double *D, const double *data)  // scft.cu:486-512
{
    FILE *out = fopen(fname.c_str(), "w");
    if (!out) return;
    fprintf(out, "# vtk DataFile Version 2.0\n");
    fprintf(out, "CT Density\n");
    fprintf(out, "ASCII\n\n");
    fprintf(out, "DATASET STRUCTURED_POINTS\n");
    fprintf(out, "DIMENSIONS %d %d %d\n", m[2], m[1], m[0]);
    fprintf(out, "ORIGIN 0.000000 0.000000 0.000000\n");
    fprintf(out, "SPACING %lf %lf %lf\n\n", D[2] / m[2], D[1] / m[1], D[0] / m[0]);
    fprintf(out, "POINT_DATA %ld\n", (long)m[0] * m[1] * m[2]);
    fprintf(out, "SCALARS scalars float\n");
    fprintf(out, "LOOKUP_TABLE default\n\n");
    // one row per (x, y): m2 values "%.4lf\t" and a newline
    const int m2 = m[2];
    write_rows(out, (long)m[0] * m[1], [&](long row, std::string &o) {
        const double *d = data + row * m2;
        for (int z = 0; z < m2; z++) append_f(o, "%.4lf\t", d[z]);
        o.push_back('\n');
    });
    fclose(out);
}

void write_win(const std::string &fn, const double *w, long M)  // scft.cu:785-788
{
    FILE *out = fopen(fn.c_str(), "w");
    if (!out) return;
    write_rows(out, M, [&](long r, std::string &o) {
        append_f(o, "%.6lf ", w[r]);
        append_f(o, "%.6lf\n", w[r + M]);
    });
    fclose(out);
}

#define CHECK(call)                                                                       \
    do {                                                                                  \
        scft_status _s = (call);                                                          \
        if (_s != SCFT_OK) {                                                              \
            fprintf(stderr, "%s failed: %s (%s)\n", #call, scft_status_string(_s),        \
                    ctx ? scft_last_error(ctx) : "");                                     \
            scft_destroy(ctx);                                                            \
            return 1;                                                                     \
        }                                                                                 \
    } while (0)

}  // namespace

int main(int argc, char *argv[])
{
    double chi = 30, f = 0.8, alpha = 0.1, phidb = 0, errtol_stop = 0, handover = 0;
    int N = 60, ens = 2, readwin = 1, justFE = 0, dostring = 1, strn = 48, nsterp = 4000;
    int precision = 64, batched = 1, checkpoint = 0, restart = 0, fcont = 0;
    int m[3] = {50, 50, 50}, fix[2] = {0, 0};
    double D[3] = {4, 4, 4};
    g_time0 = time(nullptr);
    scft_ctx *ctx = nullptr;
    std::signal(SIGINT, on_sigint);
    printf("Testing MPI: procid %d/%d\n", 0, 1);
    std::string finc = argc > 1 ? argv[1] : "input.dat";
    if (fexist(finc)) {
        printf("Reading input from %s\n\n", finc.c_str());
        auto P = read_parameters(finc);
        auto get = [&](const char *k, auto &dst) {
            auto it = P.find(k);
            if (it != P.end() && !it->second.empty()) dst = (std::remove_reference_t<decltype(dst)>)it->second.front();
        };
        get("chi", chi);
        get("f", f);
        get("N", N);
        get("alpha", alpha);
        get("readwin", readwin);
        get("ens", ens);
        get("phidb", phidb);
        get("justFE", justFE);
        get("dostring", dostring);
        get("strn", strn);
        get("nsterp", nsterp);
        get("precision", precision);
        get("batched", batched);
        get("errtol", errtol_stop);
        get("handover", handover);
        get("checkpoint", checkpoint);
        get("restart", restart);
        get("fcont", fcont);
        if (P.count("m"))
            for (size_t i = 0; i < P["m"].size() && i < 3; i++) m[i] = (int)P["m"][i];
        if (P.count("D"))
            for (size_t i = 0; i < P["D"].size() && i < 3; i++) D[i] = P["D"][i];
        if (P.count("fix"))
            for (size_t i = 0; i < P["fix"].size() && i < 2; i++) fix[i] = (int)P["fix"][i];
    } else {
        printf("%s not found. Using default values for inputs.\n", finc.c_str());
    }
    printf("chi=%g f=%g N=%d alpha=%g ens=%d phidb=%g m=%d %d %d D=%g %g %g fix=%d %d strn=%d "
           "precision=FP%d %s\n",
           chi, f, N, alpha, ens, phidb, m[0], m[1], m[2], D[0], D[1], D[2], fix[0], fix[1], strn,
           precision, batched ? "batched" : "plain");
    const long M = (long)m[0] * m[1] * m[2];

    // fields: win files (scft.cu:1057-1078) or the membrane-like start (scft.cu:1079-1098)
    std::vector<std::vector<double>> W(strn, std::vector<double>(2 * M, 0.0));
    int springsteps = 0, cpto0 = 0;
    if (readwin == 1) {
        for (int ii = 0; ii < strn; ii++) {
            std::string winf = "win" + std::to_string(ii);
            int nl = fexist(winf) ? count_lines(winf) : -1;
            if (nl == M) {
                FILE *in = fopen(winf.c_str(), "r");
                for (long r = 0; r < M; r++)
                    if (fscanf(in, "%lf %lf", &W[ii][r], &W[ii][r + M]) != 2) break;
                fclose(in);
                printf("win%d read.\n", ii);
            } else {
                printf("win%d is too small: %d.\n", ii, nl);
                springsteps += 1;
                if (ii != 0)
                    W[ii] = W[ii - 1];
                else
                    cpto0 = 1;
            }
        }
        if (cpto0 == 1 && strn > 1) W[0] = W[1];
    } else {
        for (int x = 0; x < m[0]; x++)
            for (int y = 0; y < m[1]; y++)
                for (int z = 0; z < m[2]; z++) {
                    long r = ((long)x * m[1] + y) * m[2] + z;
                    double rr = std::sqrt((z - m[2] / 2.0) * (z - m[2] / 2.0) + (y - m[1] / 2.0) * (y - m[1] / 2.0));
                    W[0][r] += -0.5 * chi * std::exp(-1.0 * std::pow((rr - m[1] / 4.0) / 8.0, 2.0));
                    W[0][r] += -0.5 * chi * std::exp(-1.0 * std::pow((rr - m[1] / 8.0) / 8.0, 2.0));
                }
    }

    scft_problem p{};
    for (int i = 0; i < 3; i++) {
        p.m[i] = m[i];
        p.D[i] = D[i];
    }
    p.N = N;
    p.alpha = alpha;
    p.ens = ens;
    p.phidb = phidb;
    p.chi = chi;
    p.f = f;
    p.strn = strn;
    p.fix[0] = fix[0];
    p.fix[1] = fix[1];
    p.dostring = dostring;
    p.springsteps = springsteps;
    p.precision = precision == 32 ? SCFT_FP32 : SCFT_FP64;
    p.batched = batched;
    p.device = 0;
    p.fcont = fcont;
    if (const char *dry = std::getenv("SCFT_DRY_RUN"); dry && dry[0] == '1') {
        // the resolved input and the start fields, then exit before any device
        // call: the input handling checked without a GPU
        printf("dryrun problem m=%d %d %d D=%.17g %.17g %.17g N=%d alpha=%.17g ens=%d phidb=%.17g chi=%.17g "
               "f=%.17g strn=%d fix=%d %d dostring=%d springsteps=%d precision=%d batched=%d fcont=%d\n",
               m[0], m[1], m[2], D[0], D[1], D[2], N, alpha, ens, phidb, chi, f, strn, fix[0], fix[1], dostring,
               springsteps, precision, batched, fcont);
        printf("dryrun run readwin=%d justFE=%d nsterp=%d errtol=%.17g checkpoint=%d restart=%d handover=%.17g\n",
               readwin, justFE, nsterp, errtol_stop, checkpoint, restart, handover);
        for (int ii = 0; ii < strn; ii++) {
            double sm = 0, sp = 0;
            for (long r = 0; r < M; r++) {
                sm += W[ii][r];
                sp += W[ii][r + M];
            }
            printf("dryrun field %d %.17g %.17g %.17g %.17g\n", ii, W[ii][0], W[ii][M], sm, sp);
        }
        return 0;
    }
    CHECK(scft_create(&p, &ctx));
    for (int ii = 0; ii < strn; ii++) CHECK(scft_set_fields(ctx, ii, W[ii].data()));
    if (restart == 1 && fexist("fields.ckpt")) {
        CHECK(scft_load_checkpoint(ctx, "fields.ckpt"));
        printf("fields.ckpt read.\n");
    }
    printf("Setup\n");

    std::vector<double> conc(4 * M), w(2 * M), FEs(strn), phctot(strn), alf(strn), errs(strn), errs3(strn);
    std::vector<int> doiis(strn), k0(strn);
    auto dump = [&](int ii, bool cb, bool win) -> int {
        double lnQ, phis[5];
        CHECK(scft_get_conc(ctx, ii, conc.data(), &lnQ, phis));
        tovtk("rhoA_" + std::to_string(ii) + ".vtk", m, D, conc.data());
        if (cb) tovtk("rhocB_" + std::to_string(ii) + ".vtk", m, D, conc.data() + 3 * M);
        if (win) {
            CHECK(scft_get_fields(ctx, ii, w.data()));
            write_win("win" + std::to_string(ii), w.data(), M);
        }
        return 0;
    };
    auto write_fes = [&]() -> int {  // scft.cu:843-850
        double FE;
        CHECK(scft_last_free_energy(ctx, &FE, FEs.data(), nullptr, nullptr, phctot.data(), alf.data()));
        FILE *out = fopen("FEs", "w");
        if (out) {
            for (int ii = 0; ii < strn; ii++)
                fprintf(out, "%lf\t%.10lf\t%.10lf\n", alf[ii] / alf[strn - 1], FEs[ii], phctot[ii]);
            fclose(out);
        }
        return 0;
    };

    // W+ relaxation of every replica before the string (scft.cu:1105-1117)
    CHECK(scft_solve_field0_all(ctx, 5000, 1e-4, k0.data()));
    CHECK(scft_get_doiis(ctx, doiis.data()));
    for (int ii = 0; ii < strn; ii++)
        if (doiis[ii] == 1 && dump(ii, true, true)) return 1;

    if (justFE != 1) {
        const double errTol = 1e-3;
        const int skip = 50;
        printf("Solving fields with %d springsteps. (procid=0)\n", springsteps);
        CHECK(scft_string_begin(ctx, -1, nsterp, errTol));
        double FEprev = 0;
        bool fp32_phase = p.precision == SCFT_FP32 && handover > 0;
        double best = 1e300;
        int best_k = 0;
        for (;;) {
            scft_iter_report rep;
            int done = 0;
            CHECK(scft_string_step(ctx, &rep, errs.data(), errs3.data(), &done));
            const int k = rep.k;
            const bool out = (k % skip == 0 || k == nsterp - 1 || g_sig == 7 ||
                              (errtol_stop > 0 && rep.errtot <= errtol_stop));
            if (out) {  // scft.cu:760-776
                auto e3 = [&](int i) { return (i >= 0 && i < strn) ? errs3[i] : 0.0; };
                printf("error  %5d/%d %.4lE/%.1lE %.2lg.\tEs: %.2lE %.2lE ... %.2lE ... %.2lE %.2lE... "
                       "%.2lg.. %.1lf (Time: %s)\n",
                       k, nsterp, rep.errtot, errTol, rep.lambda, e3(0), e3(1), e3(strn / 2), e3(strn - 2),
                       e3(strn - 1), rep.fitup, rep.stepav, tistr().c_str());
                FILE *cf = fopen("check", "w");
                if (cf) {
                    fprintf(cf, "%d %lf %lf %lf\n", k, 0.0, rep.lambda, FEprev);
                    for (int ii = 0; ii < strn; ii++) fprintf(cf, "%d %.12lf %.12lf\n", ii, errs[ii], errs3[ii]);
                    fprintf(cf, "\n");
                    fclose(cf);
                }
            }
            if (rep.did_freee) {  // scft.cu:778-791
                FEprev = rep.FE;
                if (write_fes()) return 1;
                CHECK(scft_get_doiis(ctx, doiis.data()));
                for (int ii = 0; ii < strn; ii++)
                    if (doiis[ii] == 1 && dump(ii, false, true)) return 1;
                if (checkpoint == 1) CHECK(scft_save_checkpoint(ctx, "fields.ckpt"));
            }
            if (g_sig == 7) {
                printf("Time's up (procid=0).\n");
                break;
            }
            if (errtol_stop > 0 && rep.errtot <= errtol_stop) break;
            if (done) break;
            if (fp32_phase) {
                if (rep.errtot < 0.99 * best) {
                    best = rep.errtot;
                    best_k = k;
                }
                if (rep.errtot <= handover || k - best_k >= 200) {
                    // the same run continues in FP64 from iteration k + 1
                    int kk = 0;
                    CHECK(scft_string_end(ctx, &kk));
                    scft_problem p64 = p;
                    p64.precision = SCFT_FP64;
                    scft_ctx *c64 = nullptr;
                    CHECK(scft_create(&p64, &c64));
                    scft_status hs = scft_copy_fields(c64, ctx);
                    scft_destroy(ctx);
                    ctx = c64;
                    CHECK(hs);
                    CHECK(scft_string_resume(ctx, -1, nsterp, errTol, k + 1));
                    printf("handover to FP64 at iteration %d, errtot %.4lE (Time: %s)\n", k + 1, rep.errtot,
                           tistr().c_str());
                    fp32_phase = false;
                }
            }
        }
        int kk = 0;
        CHECK(scft_string_end(ctx, &kk));
        printf("Fields solved (0) (Time: %s)\n", tistr().c_str());
    }
    // final free energy (scft.cu:1132) and outputs (scft.cu:1138-1155)
    double FE = 0;
    CHECK(scft_free_energy(ctx, &FE, nullptr, nullptr, nullptr, nullptr, nullptr));
    if (write_fes()) return 1;
    printf("Free energy caculated (procid = 0) (Time: %s)\n", tistr().c_str());
    if (FE == FE) {
        CHECK(scft_get_doiis(ctx, doiis.data()));
        for (int ii = 0; ii < strn; ii++)
            if (doiis[ii] == 1 && dump(ii, true, true)) return 1;
        if (checkpoint == 1) CHECK(scft_save_checkpoint(ctx, "fields.ckpt"));
    }
    printf("vtks and wins printed\n");
    scft_destroy(ctx);
    printf("Done (0) (Time: %s)\n", tistr().c_str());
    return 0;
}
