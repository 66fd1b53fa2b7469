"""The claim order of the persistent step kernel (csrc/step_order.cuh),
built for the host: every (phase, group, unit) item appears exactly once, and
every item comes after all items of the previous phase of its own group --
the property that keeps the kernel free of deadlock without assuming that
its CTAs are co-resident (an item waits only for items claimed before it, by
CTAs that are running or done).  No GPU."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = r"""
#include "../scft_string_b200/csrc/step_order.cuh"
extern "C" int h_step_item(int it, int G, const int *per, int *out)
{
    int p, g, u;
    if (!scft::step_item(it, G, per, p, g, u)) return 0;
    out[0] = p; out[1] = g; out[2] = u;
    return 1;
}
"""


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    from test_reg64_host import _cuda_include
    inc = _cuda_include()
    if inc is None or shutil.which("g++") is None:
        pytest.skip("needs g++ and the CUDA headers")
    d = tmp_path_factory.mktemp("step_order")
    (d / "so.cpp").write_text(SRC.replace("../scft_string_b200", os.path.join(os.path.dirname(HERE), "scft_string_b200")))
    out = str(d / "libso.so")
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I" + inc, "-o", out, str(d / "so.cpp")],
                   check=True)
    L = C.CDLL(out)
    L.h_step_item.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    return L


@pytest.mark.parametrize("G,per", [(32, (66, 64, 66, 64)), (2, (33, 64, 33, 64)), (7, (5, 3, 5, 3)),
                                   (1, (1, 1, 1, 1)), (16, (132, 64, 132, 64))])
def test_order_covers_every_item_after_its_dependencies(lib, G, per):
    perc = (C.c_int * 4)(*per)
    out = (C.c_int * 3)()
    order = []
    it = 0
    while lib.h_step_item(it, G, perc, out):
        order.append(tuple(out))
        it += 1
    total = G * sum(per)
    assert len(order) == total and len(set(order)) == total
    pos = {x: i for i, x in enumerate(order)}
    for (p, g, u), i in pos.items():
        assert 0 <= p < 4 and 0 <= g < G and 0 <= u < per[p]
        if p > 0:
            assert all(pos[(p - 1, g, v)] < i for v in range(per[p - 1]))
