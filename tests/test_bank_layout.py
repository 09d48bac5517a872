"""The stage kernel's shared-memory layout constants against the bank model.

tests/bank_model.py (beside this file) counts the shared-memory wavefronts of the stage
kernel's passes; csrc/dg_stage.cuh holds the point-array strides
(qs_stride), the per-pass task orders (TaskOrd) and the rotated coefficient
rows at p = 3 (Lay::cw). These CPU tests compile a host probe of the header
with nvcc (no GPU needed), check that the model's copy of the constants is the
header's, and that the committed choice is the model's optimum.
"""
import json
import os
import shutil
import subprocess

import pytest

import bank_model as bm

PROBE = r"""
#include "dg_stage.cuh"
#include <cstdio>
template <int P, int B> void orders() {
    using O = dgk::TaskOrd<P, B>;
    std::printf("{\"p\": %d, \"bytes\": %d, \"qs\": %d, \"x\": %d, \"y\": %d, \"z\": %d, \"zc\": %d, "
                "\"yc\": %d, \"xc\": %d, \"gather\": %d, \"minvx\": %d, \"minvy\": %d, \"minvxg\": %d}\n",
                P, B, dgk::qs_stride(P, B), O::x, O::y, O::z, O::zc, O::yc, O::xc, O::gather, O::minvx, O::minvy,
                O::minvxg);
}
int main() {
    orders<2, 8>(); orders<2, 4>(); orders<3, 8>(); orders<3, 4>();
    orders<4, 8>(); orders<4, 4>(); orders<5, 8>(); orders<5, 4>();
    std::printf("{\"cw3\": [");
    for (int b = 0; b < 64; ++b) std::printf("%d%s", dgk::Lay<3, 1>::cwl(b), b < 63 ? ", " : "");
    std::printf("]}\n");
    return 0;
}
"""

CASES = [(p, w) for p in (2, 3, 4, 5) for w in (8, 4)]


@pytest.fixture(scope="module")
def header(tmp_path_factory):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("probe")
    src, exe = d / "probe.cu", d / "probe"
    src.write_text(PROBE)
    root = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dg-mpi_b200")
    subprocess.run(["nvcc", "-std=c++17", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets",
                    "-I" + root + "/csrc", "-I" + root + "/../include", "-o", str(exe), str(src)],
                   check=True, capture_output=True)
    lines = [json.loads(l) for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                    text=True).stdout.splitlines()]
    return {(d["p"], d["bytes"]): d for d in lines if "p" in d}, lines[-1]["cw3"]


@pytest.mark.parametrize("p,w", CASES)
def test_model_tables_are_the_headers(header, p, w):
    consts, _ = header
    h = consts[(p, w)]
    assert bm.qs_stride(p, w) == h["qs"]
    o = bm.task_orders(p, w)
    assert o["x"] == bm.order2(h["x"], ("v", "byz"))
    assert o["y"] == bm.order3(h["y"], ("v", "qx", "bz"))
    assert o["z"] == bm.order2(h["z"], ("qxy", "v"))
    assert o["zc"] == bm.order2(h["zc"], ("qxy", "v"))
    assert o["yc"] == bm.order3(h["yc"], ("v", "qx", "bz"))
    assert o["xc"] == bm.order2(h["xc"], ("v", "byz"))
    assert o["gather"] == bm.order2(h["gather"], ("b", "v"))
    assert o["minvx"] == bm.order2(h["minvx"], ("v", "byz"))
    assert o["minvy"] == bm.order3(h["minvy"], ("v", "bx", "bz"))
    assert o["minvxg"] == bm.order2(h["minvxg"], ("v", "byz"))


def test_rotated_rows_are_the_headers(header):
    _, cw3 = header
    w = bm.coef_word(3, True)
    assert cw3 == [w(b % 4, (b // 4) % 4, b // 16) for b in range(64)]
    assert sorted(cw3) == list(range(64))


@pytest.mark.parametrize("p,w", CASES)
def test_committed_layout_is_the_model_optimum(p, w):
    committed = sum(c[0] for c in bm.count(p, w).values())
    best, _, _ = bm.search(p, w)
    assert committed == best


@pytest.mark.parametrize("p,w", CASES)
def test_folded_lift_gather_order_is_the_model_optimum(p, w):
    """Launch option MG: the inverse mass's x pass with the lift gather in it
    takes the model's best task order, and has fewer wavefronts than the two
    passes it replaces."""
    N, M = p + 1, p + 2
    VS, X1S, FS = (N ** 3) | 1, (N * N * M) | 1, (M * M) | 1
    ps = bm.passes(p, w, VS, X1S, bm.qs_stride(p, w), FS, bm.coef_word(p, True))
    dims, acc = ps["minvxg"]
    committed = bm.pass_cost(dims, bm.task_orders(p, w)["minvxg"], acc)[0]
    assert committed == min(bm.pass_cost(dims, o, acc)[0] for o in (("v", "byz"), ("byz", "v")))
    cur = bm.count(p, w)
    assert committed < cur["gather"][0] + cur["minvx"][0]


def test_p3_fp64_wavefront_counts():
    cur = bm.count(3, 8)
    plain = bm.count(3, 8, QS=125, orders=bm.task_orders(0, 8), rotated=False)
    assert sum(c[0] for c in cur.values()) == 1324
    assert sum(c[0] for c in plain.values()) == 1734
    assert sum(c[1] for c in cur.values()) == 1139
    assert sum(c[0] for c in bm.count(3, 8, mg=True).values()) == 1284
    # the rotated rows make every coefficient-block pencil pass conflict-free
    for name in ("minvx", "minvy", "upd"):
        assert cur[name][0] == cur[name][1]
