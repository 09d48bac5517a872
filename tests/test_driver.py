"""The C++ driver dg_solve: the reference's TOML deck and driver shape on top
of the C ABI (CPU: deck parsing and input errors; GPU: the reference's 3D
vortex regression deck run end to end through the driver)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG

SOLVE = os.path.join(PKG, "_build", "dg_solve")
EXAMPLES = os.path.join(PKG, "examples")


def run(args, **kw):
    return subprocess.run([SOLVE] + args, capture_output=True, text=True, timeout=kw.pop("timeout", 120), **kw)


@pytest.mark.parametrize("deck", sorted(f for f in os.listdir(EXAMPLES) if f.endswith(".toml")))
def test_example_decks_parse(deck):
    r = run(["-input", os.path.join(EXAMPLES, deck), "-check"])
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("case: ")


@pytest.mark.parametrize("bad,msg", [
    ('convective_flux_fcn = "Roe"', "unknown convective_flux_fcn"),
    ('basis = "LegendreHex"', "not on the device path"),
    ('type = "RK3"', "type must be FE or RK4"),
])
def test_driver_rejects_unsupported_input(tmp_path, bad, msg):
    text = open(os.path.join(EXAMPLES, "vortex3d_regression.toml")).read()
    key = bad.split("=")[0].strip()
    text = re.sub(r"^%s\s*=.*$" % key, bad, text, flags=re.M)
    deck = tmp_path / "deck.toml"
    deck.write_text(text)
    r = run(["-input", str(deck), "-check"])
    assert r.returncode == 2 and msg in r.stderr


@pytest.mark.gpu
def test_driver_reproduces_reference_regression(golden):
    r = run(["-input", os.path.join(EXAMPLES, "vortex3d_regression.toml")], timeout=300)
    assert r.returncode == 0, r.stderr
    err = {int(m.group(1)): float(m.group(2)) for m in re.finditer(r"norm_total_error\((\d)\)=(\S+)", r.stdout)}
    ref = np.array(golden["vortex3d_regression"]["l2_errors"])
    assert "number of iterations = 1000" in r.stdout
    for s in (0, 1, 3, 4):
        assert abs(err[s] - ref[s]) <= 1e-12 * ref[s], (s, err[s], ref[s])
