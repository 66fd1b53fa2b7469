// Host build of the register-resident 64-point transforms and slab phases
// (scft_string_b200/csrc/reg64.cuh) for tests/test_reg64_host.py: the warp's
// 32 lanes run one after another, phase by phase, on separate real and
// complex tiles (the device aliases them; its __syncwarp between the loads
// and the stores of a phase makes that equivalent).
#include <cstring>
#include <vector>

#include "../scft_string_b200/csrc/reg64.cuh"

using namespace scft::reg64;

extern "C" {

// 64-point FFT of x (64 complex as 128 floats) in place; pin: permuted-input variant
void h_fft64(int sign, int pin, float *x)
{
    float2 *v = reinterpret_cast<float2 *>(x);
    if (pin)
        sign < 0 ? fft64_pin<-1>(v) : fft64_pin<+1>(v);
    else
        sign < 0 ? fft64<-1>(v) : fft64<+1>(v);
}

int h_perm(int k) { return perm(k); }

// real slab [64 y][64 z] -> half spectrum [64 ky][33 kz] (complex as float pairs)
void h_slab_forward(const float *real, float *spec)
{
    std::vector<float> R(kTileFloats, 0.f);
    std::vector<float2> T(kTileFloats / 2);
    for (int y = 0; y < 64; y++)
        for (int z = 0; z < 64; z++) R[y * kRowPitch + z] = real[y * 64 + z];
    std::vector<float2> v(32 * 64);
    for (int p = 0; p < 32; p++) fz_load(R.data(), p, &v[p * 64]);
    for (int p = 0; p < 32; p++) fz_fft_store(T.data(), p, &v[p * 64]);
    for (int kz = 0; kz < 32; kz++) fy(T.data(), kz, &v[kz * 64], reinterpret_cast<float2 *>(spec));
}

// half spectrum [64 ky][33 kz] -> real slab [64 y][64 z] (unnormalised)
void h_slab_inverse(const float *spec, float *real)
{
    std::vector<float> R(kTileFloats, 0.f);
    std::vector<float2> T(kTileFloats / 2);
    std::vector<float2> v(32 * 64);
    for (int kz = 0; kz < 32; kz++) iy(reinterpret_cast<const float2 *>(spec), kz, &v[kz * 64], T.data());
    for (int p = 0; p < 32; p++) iz_load(T.data(), p, &v[p * 64]);
    for (int p = 0; p < 32; p++) iz_fft_store(R.data(), p, &v[p * 64]);
    for (int y = 0; y < 64; y++)
        for (int z = 0; z < 64; z++) real[y * 64 + z] = R[y * kRowPitch + z];
}
}
