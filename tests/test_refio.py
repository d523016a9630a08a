"""Reference case directories, restart and monitor files (host side, no GPU).

Pins: the delivered cases' Config.ini assignments (fixture `case_namelists`) must load as exactly the
cases the GPU tests run; the mesh and velocity writers must reproduce the delivered files byte for
byte (fixture SHA-256); sparse_residual.csv rows must reproduce the reference's own lines character
for character from their values.  The rest are round trips and the reference's rejection rules.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from ugks2d_high_order_b200 import refio
from ugks2d_high_order_b200.case import (batched_cases, load_velocity_half32, reference_case,
                                         refined_high_order_case, velocity_table)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
METHOD = {"low_explicit": "Explicit", "low_implicit": "ImplicitSteady", "high_implicit": "HighOrderImplicit"}


def golden():
    with open(os.path.join(GOLDEN, "reference_golden.json")) as f:
        return json.load(f)


def mesh():
    g = np.load(os.path.join(GOLDEN, "mesh_8x64.npy"))
    return g[0], g[1]


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def test_namelist_parser_reads_fortran_forms():
    text = """! leading comment with & and / characters
&config_para
  A = 1.5d0, B = -2 ! trailing comment
  S = 'it''s ! not a comment / nor an end'
  L1 = .true.   L2 = F
  ARR = 10 10 2 2
  REP = 3*0.5d-1
  WallUx(3) = -3.0d0
  WallUx(4) = 3.0D0
/
&boundary_para X = 7 /
$DIS_para
0
$DIS_para
"""
    g = refio.parse_namelists(text)
    c, b = g["config_para"], g["boundary_para"]
    assert c.get("a") == 1.5 and c.get("b") == -2
    assert c.get("s") == "it's ! not a comment / nor an end"
    assert c.get("l1") is True and c.get("l2") is False
    assert c.get_array("arr", 4, [0] * 4) == [10, 10, 2, 2]
    assert c.get_array("rep", 3, [0] * 3) == [0.05, 0.05, 0.05]
    assert c.get_array("wallux", 4, [0.0] * 4) == [0.0, 0.0, -3.0, 3.0]
    assert b.get("x") == 7
    with pytest.raises(refio.CaseError):
        refio.parse_namelists("&config_para\n A = 1\n")


def config_text(name):
    """Config.ini of a delivered case, rebuilt from its fixture assignments."""
    nml = golden()["case_namelists"][name]
    return "\n".join(f"&{g}\n" + "\n".join(f"{k} = {' '.join(v)}" for k, v in kv.items()) + "\n/"
                      for g, kv in nml.items()) + "\n"


@pytest.mark.parametrize("name", ["low_explicit", "low_implicit", "high_implicit"])
def test_delivered_namelists_load_as_the_reference_cases(name):
    case = refio.case_from_config(refio.parse_namelists(config_text(name)), mesh())
    assert case == reference_case(METHOD[name])


@pytest.mark.parametrize("name", ["low_explicit", "low_implicit", "high_implicit"])
def test_reference_case_directories_load_unchanged(name, tmp_path):
    """A delivered case directory (the three share one Mesh2d.dat and one velocity file): the binary
    files are written by the writers and checked against the delivered files' SHA-256, Config.ini
    holds the delivered assignments; load_case_dir gives the case the GPU tests run."""
    want = golden()["case_file_sha256"]
    gx, gy = mesh()
    refio.write_mesh(str(tmp_path / "Mesh2d.dat"), gx, gy)
    u, v, w = load_velocity_half32()
    refio.write_velocity_file(str(tmp_path / "velocity_half32_scale2.dat"), u, v, w, 32, 32)
    for f in ("Mesh2d.dat", "velocity_half32_scale2.dat"):
        assert sha(tmp_path / f) == want[f]
    (tmp_path / "Config.ini").write_text(config_text(name))
    d = refio.load_case_dir(str(tmp_path))
    assert d.case == reference_case(METHOD[name])
    for x, y in zip((d.u, d.v, d.w), load_velocity_half32()):
        assert np.array_equal(x, y)
    assert d.run["Iflag_InitFlow"] == 0 and d.run["MAX_ITER"] == d.case.max_iter


def test_mesh_and_velocity_writers_reproduce_the_delivered_files(tmp_path):
    want = golden()["case_file_sha256"]
    gx, gy = mesh()
    refio.write_mesh(str(tmp_path / "Mesh2d.dat"), gx, gy)
    assert sha(tmp_path / "Mesh2d.dat") == want["Mesh2d.dat"]
    u, v, w = load_velocity_half32()
    refio.write_velocity_file(str(tmp_path / "vel.dat"), u, v, w, 32, 32)
    assert sha(tmp_path / "vel.dat") == want["velocity_half32_scale2.dat"]
    gx2, gy2 = refio.read_mesh(str(tmp_path / "Mesh2d.dat"), 8, 64)
    assert np.array_equal(gx2, gx) and np.array_equal(gy2, gy)
    assert refio.mesh_spacing(gx, gy) == (0.125, 1.0 / 64.0)
    with pytest.raises(refio.CaseError) as e:
        refio.read_mesh(str(tmp_path / "Mesh2d.dat"), 8, 32)
    assert e.value.reference_code == 474


def test_velocity_file_checks_follow_the_reference(tmp_path):
    u, v, w = load_velocity_half32()
    p = str(tmp_path / "vel.dat")
    with pytest.raises(refio.CaseError) as e:
        refio.read_velocity_file(p, 32, 32)
    assert e.value.reference_code == 201
    refio.write_velocity_file(p, u, v, w, 32, 32)
    with pytest.raises(refio.CaseError) as e:
        refio.read_velocity_file(p, 16, 16)
    assert e.value.reference_code == 203
    w2 = w.copy()
    w2[5] *= 1.0 + 1e-15                                    # breaks the mirror symmetry of the weights
    refio.write_velocity_file(p, u, v, w2, 32, 32)
    with pytest.raises(refio.CaseError) as e:
        refio.read_velocity_file(p, 32, 32)
    assert e.value.reference_code == 205
    with open(p, "w") as f:
        f.write("32 32\n1.0 2.0\n")
    with pytest.raises(refio.CaseError) as e:
        refio.read_velocity_file(p, 32, 32)
    assert e.value.reference_code == 204


def test_case_directory_round_trip(tmp_path):
    cases = [(reference_case(m), 32) for m in ("Explicit", "ImplicitSteady", "HighOrderImplicit")]
    cases.append((refined_high_order_case(), 48))
    cases += [(c, n) for c, n in batched_cases(4)]
    for k, (case, n) in enumerate(cases):
        d = str(tmp_path / f"case{k}")
        u, v, w = velocity_table(n)
        refio.write_case_dir(d, case, u, v, w)
        got = refio.load_case_dir(d)
        assert got.case == case, k
        for x, y in zip((got.u, got.v, got.w), (u, v, w)):
            assert np.array_equal(x, y)


def test_unsupported_settings_are_refused():
    nml = golden()["case_namelists"]["low_implicit"]

    def load(**over):
        kv = {g: dict(v) for g, v in nml.items()}
        for key, val in over.items():
            grp = "boundary_para" if key in ("BC_Type", "ACC") else "config_para"
            kv[grp][key] = val.split()
        text = "\n".join(f"&{g}\n" + "\n".join(f"{k} = {' '.join(v)}" for k, v in x.items()) + "\n/"
                         for g, x in kv.items())
        return refio.case_from_config(refio.parse_namelists(text), mesh())

    load()
    for key, val in (("NP_X", "2"), ("BC_Type", "10 10 3 3"), ("Implicit_MaxRetries", "8"),
                     ("Implicit_MicroSweeps", "2"), ("flag_vislaw", "2"), ("ACC", "0.5d0"),
                     ("TimeIntegration_method", "'S2Steady'"), ("NP_Y", "7")):
        with pytest.raises(refio.CaseError):
            load(**{key: val})


def _state(nx, ny, nv, seed):
    rng = np.random.default_rng(seed)
    return rng.random((nx * ny, 4)), rng.random((nx * ny, nv)), rng.random((nx * ny, nv))


def test_restart_files_round_trip(tmp_path):
    nx, ny, nv = 8, 16, 36
    W, h, b = _state(nx, ny, nv, 1)
    gx, gy = refio.cartesian_mesh(nx, ny)
    refio.write_restart(str(tmp_path), W, h, b, nx, ny, gx, gy)
    W2, h2, b2 = refio.read_restart(str(tmp_path), nx, ny, nv)
    assert np.array_equal(W, W2) and np.array_equal(h, h2) and np.array_equal(b, b2)
    recs = refio.read_records(str(tmp_path / "flow2d.dat"))
    assert [len(r) for r in recs] == [4, 12, 8 * 4 * nx * ny]
    # column-major: the first values of the data record are rho of cells (1,1), (2,1), ...
    assert np.array_equal(np.frombuffer(recs[2], "<f8")[:nx], W[:nx, 0])
    recs = refio.read_records(str(tmp_path / "vdf2d.dat"))
    vals = np.frombuffer(recs[2], "<f8")
    assert np.array_equal(vals[: nx * ny], h[:, 0]) and np.array_equal(vals[nv * nx * ny: nv * nx * ny + 1], b[:1, 0])
    with pytest.raises(refio.CaseError):
        refio.read_restart(str(tmp_path), nx, ny, nv + 1)


def test_mass_restart_round_trip_and_binding(tmp_path):
    nml = golden()["case_namelists"]["low_implicit"]
    text = "\n".join(f"&{g}\n" + "\n".join(f"{k} = {' '.join(v)}" for k, v in kv.items()) + "\n/"
                     for g, kv in nml.items())
    groups = refio.parse_namelists(text)
    u, v, w = load_velocity_half32()
    nx, ny, nv = 8, 64, 1024
    W, h, b = _state(nx, ny, nv, 2)
    ident = refio.restart_identity(groups, u, w)
    s = 0.0
    for x in w:
        s += x
    assert ident[29] == s and ident[0] == 8.0 and ident[3] == 8.0 and ident[17] == 3.872983346207417
    refio.write_mass_restart(str(tmp_path), groups, u, w, W, h, b, nx, ny, 0.984375, (1e-3, 0.0, -2e-3, 0.5), 1096)
    assert sorted(os.listdir(tmp_path)) == [f"closed_mass_rank{r}.bin" for r in range(8)]
    size = os.path.getsize(tmp_path / "closed_mass_rank0.bin")
    assert size == 6 * 4 + 36 * 8 + (8 + 4) * (8 + 4) * (4 + 2 * nv) * 8
    m0, ledger, step = refio.read_mass_restart(str(tmp_path), groups, u, w, nx, ny, nv, W, h, b)
    assert m0 == 0.984375 and step == 1096 and np.array_equal(ledger, [1e-3, 0.0, -2e-3, 0.5])
    W2 = W.copy()
    W2[100, 0] += 1e-16 * W2[100, 0] + 1e-300
    with pytest.raises(refio.CaseError):                       # bound to a different flow pair
        refio.read_mass_restart(str(tmp_path), groups, u, w, nx, ny, nv, W2, h, b)
    other = refio.parse_namelists(text.replace("CFL = 0.1d0", "CFL = 0.2d0"))
    with pytest.raises(refio.CaseError):                       # RestartIdentity mismatch
        refio.read_mass_restart(str(tmp_path), other, u, w, nx, ny, nv)


def test_sparse_rows_reproduce_the_reference_lines():
    g = golden()
    for case, lines in g["sparse_lines"].items():
        assert lines[0] == refio.SPARSE_HEADER
        for line in lines[1:]:
            parts = line.split(",")
            vals = [float(x) for x in parts[3:]]
            rep = np.array(vals[:53])
            assert vals[53] == 1.0
            assert refio.sparse_row(int(parts[0]), int(parts[1]), rep, True, parts[2]) == line


def test_residual_reference_keeps_its_epoch(tmp_path):
    p = str(tmp_path)
    refio.write_residual_reference(p, 0.4379937552164235, 0.5371654919248009, 1e-8, 1e-12)
    assert refio.read_residual_reference(p) == (0, 0.4379937552164235, 0.5371654919248009, 1e-8, 1e-12)
    text = open(tmp_path / "residual_reference.in").read()
    assert text.startswith("0   4.3799375521642347E-001   5.3716549192480090E-001 ")
    with open(tmp_path / "residual_reference.in", "w") as f:
        f.write(text.replace("0 ", "7 ", 1))
    refio.write_residual_reference(p, 1.0, 2.0, 1e-8, 1e-12)
    assert refio.read_residual_reference(p)[:3] == (7, 1.0, 2.0)


def _report_from_sparse(rows):
    """A device report vector carrying the pre-update science of step 2 (the view of accepted state 1)
    and the moment error of step 2's update (the accepted state 2's)."""
    rep = np.zeros(80)
    rep[57:79] = [rows[0][f"science_{k}"] for k in range(1, 23)]
    rep[1] = rows[1]["moment"]
    rep[53] = 1.0
    return rep


@pytest.mark.parametrize("case", ["low_implicit", "high_implicit"])
def test_implicit_stdout_line_reproduces_the_reference(case):
    g = golden()
    line = g[case + "_summary"][0]
    wall = float(line.split("wall=")[1].split()[0])
    rep = _report_from_sparse(g[case + "_sparse"])
    assert refio.implicit_stdout_line(2, rep, 1000.0, wall) == line


def test_residual_implicit_rows_follow_the_fortran_format(tmp_path):
    g = golden()
    rep = _report_from_sparse(g["low_implicit_sparse"])
    rep[55], rep[52] = 8.6528e-5, -1.25e-10
    w = refio.ResidualImplicitWriter(str(tmp_path), 1000.0, True)
    w.append(1, rep, 0.5)
    w.append(2, rep, 1.0)
    lines = open(tmp_path / "ResidualImplicit.plt").read().splitlines()
    assert lines[0] == refio.RESIDUAL_IMPLICIT_HEADER and len(lines) == 3
    row = lines[2]
    assert len(row) == 12 + 11 * 18 + 8 + 5 * 18 + 12 + 15 * 18 + 2 * 25
    assert len(lines[0].split()) - 2 == 36                      # 36 columns after "VARIABLES ="
    f = [float(row[0:12])] + [float(row[12 + 18 * k: 30 + 18 * k]) for k in range(11)]
    assert f[0] == 2 and f[1] == 8.6528e-5 and f[2] == 1000.0 and f[4] == float(f"{rep[57]:.9E}")
    assert float(row[-50:-25]) == -1.25e-10 and float(row[-25:]) == 1.0
