"""Pointwise physics of the kernels on the host (CPU only): the header
dg_physics.cuh compiles as plain C++, so a small probe evaluates its fluxes
in FP64 and FP32 beside the oracle's restatement of the reference.

The FP32 residual evaluates HLLC on states whose energy is stored relative
to a constant (flux_hllc_shift).  In exact arithmetic that is the
reference's HLLC (euler/functions.cpp:298-399) with the constant pressure
(gamma-1) E_ref times the normal left out of the momenta; in FP32 it must
keep the momenta's digits at low Mach, where rE is ~180 and P ~70.
"""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import pyoracle
from conftest import ROOT

PROBE = r"""
#include "dg_physics.cuh"
#include <cstdio>
#include <cstdlib>
// reads lines "g eref UL[5] UR[5] N[3]" and prints the flux of
// flux_hllc_n (full energy) and flux_hllc_shift (shifted energy; its momenta
// leave out the constant pressure) in FP64 and FP32
template <typename T>
void run(double g, double eref, const double* ul, const double* ur, const double* N, bool shift, double* F)
{
    T UL[5], UR[5], n[3], Fo[5];
    const double nm = std::sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    for (int d = 0; d < 3; ++d) n[d] = T(N[d] * (1.0 / nm));
    for (int s = 0; s < 5; ++s) {
        UL[s] = T(ul[s] - (shift && s == 4 ? eref : 0.0));
        UR[s] = T(ur[s] - (shift && s == 4 ? eref : 0.0));
    }
    bool ok = shift ? dgp::flux_hllc_shift<T>(T(g), UL, UR, n, T(nm), T(eref), Fo)
                    : dgp::flux_hllc_n<T>(T(g), UL, UR, n, T(nm), Fo);
    for (int s = 0; s < 5; ++s) F[s] = double(Fo[s]);
    if (!ok) F[0] = NAN;
}
int main()
{
    double g, eref, ul[5], ur[5], N[3];
    while (std::scanf("%lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf", &g, &eref, ul, ul + 1, ul + 2,
                      ul + 3, ul + 4, ur, ur + 1, ur + 2, ur + 3, ur + 4, N, N + 1, N + 2) == 15) {
        double F[4][5];
        run<double>(g, eref, ul, ur, N, false, F[0]);
        run<double>(g, eref, ul, ur, N, true, F[1]);
        run<float>(g, eref, ul, ur, N, false, F[2]);
        run<float>(g, eref, ul, ur, N, true, F[3]);
        std::printf("[");
        for (int k = 0; k < 4; ++k)
            for (int s = 0; s < 5; ++s) std::printf("%.17g%s", F[k][s], k == 3 && s == 4 ? "]\n" : ", ");
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("physics")
    src, exe = d / "probe.cpp", d / "probe"
    src.write_text(PROBE)
    subprocess.run([cxx, "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "dg-mpi_b200", "csrc"), "-o", str(exe),
                    str(src)], check=True, capture_output=True)

    def run(rows):
        text = "\n".join(" ".join(repr(float(x)) for x in r) for r in rows) + "\n"
        out = subprocess.run([str(exe)], input=text, check=True, capture_output=True, text=True).stdout
        return np.array([json.loads(l) for l in out.splitlines()]).reshape(-1, 4, 5)

    return run


def states(rng, n, mach):
    """Random face states around a flow of the given Mach number (gamma 1.4,
    rho ~ 1, |u| ~ 1, P = 1/(gamma M^2)), with the energy reference the mean
    energy of the two sides."""
    g = 1.4
    rows = []
    for _ in range(n):
        U = []
        for _side in range(2):
            rho = 1.0 + 0.1 * rng.standard_normal()
            u = rng.standard_normal(3)
            P = 1.0 / (g * mach * mach) * (1.0 + 0.05 * rng.standard_normal())
            U.append([rho, *(rho * u), P / (g - 1) + 0.5 * rho * u @ u])
        N = rng.standard_normal(3) * 0.3
        eref = 0.5 * (U[0][4] + U[1][4])
        rows.append([g, eref, *U[0], *U[1], *N])
    return rows


def test_shifted_hllc_is_reference_hllc_in_fp64(probe):
    rng = np.random.default_rng(5)
    rows = states(rng, 400, 0.3) + states(rng, 400, 2.0)  # subsonic and supersonic faces: every branch
    F = probe(rows)
    assert np.isfinite(F).all()
    # restore the constant pressure (gamma-1) E_ref |N| n_hat in the momenta
    R = np.array(rows)
    N = R[:, 12:15]
    shifted = F[:, 1].copy()
    shifted[:, 1:4] += (R[:, 0] - 1.0)[:, None] * R[:, 1][:, None] * N
    scale = np.abs(F[:, 0]).max()
    assert np.abs(shifted - F[:, 0]).max() / scale < 1e-13
    # the unshifted FP64 flux is the oracle's (the reference's HLLC)
    for r, f in zip(rows[:50], F[:50]):
        ul, ur, N = np.array(r[2:7]), np.array(r[7:12]), np.array(r[12:15])
        np.testing.assert_allclose(f[0], pyoracle.num_flux("HLLC", r[0], ul, ur, N)[0], rtol=1e-12, atol=1e-12)


def test_shifted_hllc_keeps_momentum_digits_in_fp32_at_low_mach(probe):
    rng = np.random.default_rng(9)
    F = probe(states(rng, 400, 0.1))
    mom = slice(1, 4)
    # each FP32 form against its FP64 value: the full-energy form rounds the
    # full pressure into the momenta, the shifted form only the fluctuation
    err_full = np.abs(F[:, 2, mom] - F[:, 0, mom]).max()
    err_shift = np.abs(F[:, 3, mom] - F[:, 1, mom]).max()
    # the pressure is ~70: FP32 rounding of rE ~180 costs ~1.3e-5 absolute in
    # the unshifted form; the shifted form keeps FP32's relative rounding of
    # the O(10) wave-speed terms (~2.6e-6 here)
    assert err_shift < 0.35 * err_full, (err_shift, err_full)
    assert err_shift < 5e-6
