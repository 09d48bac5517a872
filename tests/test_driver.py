"""The C++ driver dg_solve: the reference's TOML deck and driver shape on top
of the C ABI (CPU: deck parsing and input errors; GPU: the reference's 3D
vortex regression deck run end to end through the driver)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG
import dg_b200

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


def test_mutated_decks_are_refused_or_parsed_never_crash(tmp_path):
    """Seeded mutations of the example decks (deleted, truncated, shuffled and
    garbage lines, out-of-range values, unterminated strings and arrays)
    end in a clean parse (exit 0) or a refusal with a message (exit 2),
    never in a signal."""
    import random
    rng = random.Random(7)
    decks = [open(os.path.join(EXAMPLES, f)).read() for f in sorted(os.listdir(EXAMPLES)) if f.endswith(".toml")]
    junk = ['"', "]", "[", "=", " = 1e999", " = -5", ",", "\\"]
    inserts = ["[Numerics]", "order = 99", "order = -1", "data = []", "timestep = 0", "end = -1",
               'file = "nonexistent.h5"', 'type = "Bogus"', 'x = "unterminated']
    values = ['"a"', "[1,2", "1.5.5", "true", "-0", "99999999999999999999"]
    outcomes = {0: 0, 2: 0}
    for it in range(150):
        lines = rng.choice(decks).splitlines()
        for _ in range(rng.randint(1, 3)):
            k = rng.randrange(len(lines))
            op = rng.randrange(6)
            if op == 0:
                del lines[k]
            elif op == 1:
                lines[k] = lines[k][:rng.randrange(len(lines[k]) + 1)]
            elif op == 2:
                lines[k] += rng.choice(junk)
            elif op == 3:
                lines.insert(k, rng.choice(inserts))
            elif op == 4 and "=" in lines[k]:
                lines[k] = lines[k].split("=")[0] + "= " + rng.choice(values)
            else:
                lines[k] = "".join(rng.sample(lines[k], len(lines[k])))
        deck = tmp_path / f"d{it}.toml"
        deck.write_text("\n".join(lines) + "\n")
        r = run(["-input", str(deck), "-check"], cwd=str(tmp_path))
        assert r.returncode in (0, 2), (it, r.returncode, deck.read_text(), r.stderr[-500:])
        outcomes[r.returncode] += 1
    assert outcomes[2] > 50 and outcomes[0] > 10, outcomes


def _check_regression(r, golden):
    assert r.returncode == 0, r.stderr
    err = {int(m.group(1)): float(m.group(2)) for m in re.finditer(r"norm_total_error\((\d)\)=(\S+)", r.stdout)}
    ref = np.array(golden["vortex3d_regression"]["l2_errors"])
    assert "number of iterations = 1000" in r.stdout
    for s in (0, 1, 3, 4):
        assert abs(err[s] - ref[s]) <= 1e-12 * ref[s], (s, err[s], ref[s])


@pytest.mark.gpu
def test_driver_reproduces_reference_regression(golden, tmp_path):
    """No meshes/cube_4.h5 exists: the driver generates the periodic box that
    file holds; the final state goes to data.h5 as the reference writes it."""
    r = run(["-input", os.path.join(EXAMPLES, "vortex3d_regression.toml")], timeout=300, cwd=str(tmp_path))
    _check_regression(r, golden)
    assert "periodic hex" in r.stdout
    U, t = dg_b200.read_solution_h5(str(tmp_path / "data.h5"))
    assert U.shape == (64, 64, 5) and t == pytest.approx(1.0, abs=1e-12)


@pytest.mark.gpu
def test_driver_runs_reference_regression_from_a_mesh_file(golden, tmp_path):
    """The same deck on a cube_4.h5 mesh file of the reference's format (the
    4^3 box with rotated element numberings written by dg_mesh_write_h5):
    read through dg_mesh_read_h5, same published errors."""
    (tmp_path / "meshes").mkdir()
    dg_b200.write_mesh_h5(str(tmp_path / "meshes" / "cube_4.h5"),
                          dg_b200.periodic_box((4, 4, 4), (0, 0, 0), (1, 1, 1), rotate_seed=3))
    r = run(["-input", os.path.join(EXAMPLES, "vortex3d_regression.toml")], timeout=300, cwd=str(tmp_path))
    _check_regression(r, golden)
    assert "cube_4.h5 (64 hex elements, 192 interior faces)" in r.stdout


def test_driver_refuses_a_two_dimensional_mesh_file(tmp_path):
    text = open(os.path.join(EXAMPLES, "vortex3d_regression.toml")).read()
    quad = os.path.join(os.path.dirname(__file__), "golden", "meshes", "quad_2x2.h5")
    deck = tmp_path / "deck.toml"
    deck.write_text(re.sub(r"^file\s*=.*$", 'file = "%s"' % quad, text, flags=re.M))
    r = run(["-input", str(deck), "-check"])
    assert r.returncode == 2 and "takes linear hexahedra" in r.stderr


def _deck(tmp_path, name, steps, output):
    text = open(os.path.join(EXAMPLES, "vortex_xy_8cubed_p2.toml")).read()
    text = re.sub(r"^steps\s*=.*$", "steps = %d" % steps, text, flags=re.M)
    deck = tmp_path / name
    deck.write_text(text + "\n[Output]\n" + output + "\n")
    return str(deck)


def test_driver_deck_with_output_extensions_parses(tmp_path):
    r = run(["-input", _deck(tmp_path, "d.toml", 5, 'restart_file = "x.state"\njson = true'), "-check"])
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_driver_rejects_a_restart_file_of_another_mesh(tmp_path):
    bad = tmp_path / "other.state"
    np.array([7, 27, 5], np.int64).tofile(str(bad))
    r = run(["-input", _deck(tmp_path, "d.toml", 5, 'restart_file = "%s"' % bad)], cwd=str(tmp_path))
    assert r.returncode == 2 and "does not hold a state of this mesh" in r.stderr


@pytest.mark.gpu
def test_driver_checkpoint_resume_matches_unbroken_run(tmp_path):
    """20 steps in one run against 12 steps, a checkpoint, and 8 more steps
    from it: the states are bit for bit the same, and the JSON metrics line
    reports the run."""
    import json
    full, part, rest = tmp_path / "full.state", tmp_path / "part.state", tmp_path / "rest.state"
    r = run(["-input", _deck(tmp_path, "a.toml", 20, 'state_file = "%s"\njson = true' % full)], cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    metrics = json.loads(r.stdout.strip().splitlines()[-1])
    assert metrics["steps"] == 20 and metrics["stages_per_step"] == 4 and metrics["dof"] == 512 * 27 * 5
    assert len(metrics["l2_error"]) == 5 and metrics["dof_stage_per_s"] > 0
    r = run(["-input", _deck(tmp_path, "b.toml", 12, 'state_file = "%s"' % part)], cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    r = run(["-input", _deck(tmp_path, "c.toml", 8, 'restart_file = "%s"\nstate_file = "%s"' % (part, rest))],
            cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr

    def load(path):
        raw = open(path, "rb").read()
        hdr = np.frombuffer(raw[:24], np.int64)
        t = np.frombuffer(raw[24:32], np.float64)[0]
        return hdr, t, np.frombuffer(raw[32:], np.float64)
    h1, t1, u1 = load(full)
    h2, t2, u2 = load(rest)
    assert list(h1) == list(h2) == [512, 27, 5]
    assert t1 == t2 == metrics["time"]
    assert np.array_equal(u1, u2)


@pytest.mark.gpu
def test_driver_resumes_from_its_data_h5(tmp_path):
    """12 steps written to data.h5 (the writer's schema), then 8 more from that
    file, against 20 unbroken steps: bit for bit the same state and time."""
    r = run(["-input", _deck(tmp_path, "a.toml", 20, 'solution_file = "full.h5"')], cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    r = run(["-input", _deck(tmp_path, "b.toml", 12, "")], cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    r = run(["-input", _deck(tmp_path, "c.toml", 8, 'restart_file = "data.h5"\nsolution_file = "rest.h5"')],
            cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    u1, t1 = dg_b200.read_solution_h5(str(tmp_path / "full.h5"))
    u2, t2 = dg_b200.read_solution_h5(str(tmp_path / "rest.h5"))
    assert t1 == t2 and np.array_equal(u1, u2)


def test_2d_deck_with_a_quad_mesh_file_parses(tmp_path):
    quad = os.path.join(os.path.dirname(__file__), "golden", "meshes", "quad_1x1.h5")
    text = open(os.path.join(EXAMPLES, "vortex2d_box8_p2.toml")).read()
    deck = tmp_path / "deck.toml"
    deck.write_text(re.sub(r"^file\s*=.*$", 'file = "%s"' % quad, text, flags=re.M))
    r = run(["-input", str(deck), "-check"])
    assert r.returncode == 0, r.stderr
    assert "(1 quadrilaterals, 2 interior faces)" in r.stdout


@pytest.mark.gpu
def test_driver_2d_deck_reproduces_reference_convergence_entry(golden, tmp_path):
    """The reference's 2D vortex deck on the 8x8 box (p = 2): its density
    error against the convergence table to the 2D pin, and data.h5 in the
    writer's schema with four state variables."""
    from test_oracle2d import TABLE, PIN_RTOL
    r = run(["-input", os.path.join(EXAMPLES, "vortex2d_box8_p2.toml")], timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    err = {int(m.group(1)): float(m.group(2)) for m in re.finditer(r"norm_total_error\((\d)\)=(\S+)", r.stdout)}
    assert "number of iterations = 1000" in r.stdout
    assert abs(err[0] / TABLE[2][2] - 1.0) < PIN_RTOL, err[0]
    U, t = dg_b200.read_solution_h5(str(tmp_path / "data.h5"))
    assert U.shape == (64, 9, 4) and t == pytest.approx(1.0, abs=1e-12)


@pytest.mark.gpu
def test_driver_post_mode_recomputes_the_errors_of_a_run(tmp_path):
    """dg_solve -post (the reference's post tool, src/post/main.cpp:204-253):
    the deck's case, data.h5's state and time, the same L2 errors the run
    printed; 3D and 2D decks."""
    def errors(out):
        return {int(m.group(1)): m.group(2) for m in re.finditer(r"norm_total_error\((\d)\)=(\S+)", out)}
    deck3 = _deck(tmp_path, "a.toml", 7, "")
    r = run(["-input", deck3], cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    p = run(["-input", deck3, "-post", "data.h5"], cwd=str(tmp_path))
    assert p.returncode == 0, p.stderr
    assert errors(p.stdout) == errors(r.stdout) and len(errors(p.stdout)) == 5
    assert re.search(r"^time=", p.stdout, re.M)
    deck2 = os.path.join(EXAMPLES, "vortex2d_box8_p2.toml")
    (tmp_path / "two").mkdir()
    r = run(["-input", deck2], cwd=str(tmp_path / "two"), timeout=300)
    assert r.returncode == 0, r.stderr
    p = run(["-input", deck2, "-post"], cwd=str(tmp_path / "two"))
    assert p.returncode == 0, p.stderr
    assert errors(p.stdout) == errors(r.stdout) and len(errors(p.stdout)) == 4
