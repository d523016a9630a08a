"""Generate the committed golden fixtures from the reference's own case files and logs.

Run once in a container that has the reference checkout (the GPU host does not):

    python tests/golden/make_fixtures.py <the reference checkout>

Outputs (all small, committed):
  velocity_half32_scale2.npy  - the 1024-row (u, v, w) table of cases/*/velocity_half32_scale2.dat,
                                parsed to float64 exactly (18 significant digits in the file).
  mesh_8x64.npy               - gridx, gridy node arrays decoded from cases/*/Mesh2d.dat
                                (Fortran unformatted, records "9 65" then gridx, gridy).
  reference_golden.json       - numbers the reference itself printed for this hot path, and its case inputs:
     * low_explicit 2-step `dtPhysical` and `res:` line  (docs/release_checks/low_explicit/stdout.log)
     * low_implicit / high_implicit sparse_residual.csv rows  (docs/release_checks/*/sparse_residual.csv)
     * the implicit "Implicit iter=2 ..." summary lines        (docs/release_checks/*/stdout.log)
     * converged 64-point profiles of the three methods        (docs/couette_results/profiles_three_methods.plt)
     * static-equilibrium residual / update maxima             (checks/VERIFICATION.json)
     * end-of-run summaries of the explicit and implicit runs  (docs/couette_results/analysis.json):
       step count, final selected residuals, c_final, per-wall native pnn/pnt/qn
     * the namelist assignments of cases/*/Config.ini as raw tokens   (case_namelists)
     * SHA-256 of cases/low_implicit/Mesh2d.dat and the velocity file  (case_file_sha256)
     * the text lines of docs/release_checks/*/sparse_residual.csv     (sparse_lines)
"""
import json
import os
import re
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_velocity(path):
    with open(path) as f:
        n1, n2 = (int(t) for t in f.readline().split())
        rows = [tuple(float(t.replace("D", "E")) for t in f.readline().split()) for _ in range(n1 * n2)]
    return n1, n2, np.array(rows, dtype=np.float64)


def read_mesh(path):
    with open(path, "rb") as f:
        data = f.read()
    # record 1: two int32 (Nx_all+1, Ny_all+1)
    (l1,) = struct.unpack_from("<i", data, 0)
    nx0, ny0 = struct.unpack_from("<ii", data, 4)
    off = 4 + l1 + 4
    (l2,) = struct.unpack_from("<i", data, off)
    vals = np.frombuffer(data, dtype="<f8", count=l2 // 8, offset=off + 4)
    gx = vals[: nx0 * ny0].reshape(ny0, nx0)  # Fortran (i,j) column-major -> [j][i]
    gy = vals[nx0 * ny0:].reshape(ny0, nx0)
    return nx0, ny0, gx.copy(), gy.copy()


def parse_velocity_tables(path):
    """raw_node / raw_weight of the half16 and half32 rules (mod_VelocityTables.f90:40-96)."""
    import re
    txt = open(path).read()
    out = {}
    for name in ("half16", "half32"):
        body = txt[txt.index("case('%s')" % name):]
        body = body[:body.index("case(", 5) if "case(" in body[5:] else body.index("end select")]
        arrays = {}
        for key in ("raw_node", "raw_weight"):
            seg = body[body.index(key + "=["):]
            seg = seg[:seg.index("]")]
            arrays[key] = [float(x.replace("_KREAL", "").replace("d", "e"))
                           for x in re.findall(r"[-+]?\d\.\d+e[-+]\d+_KREAL", seg)]
        out[name] = arrays
    out["source"] = "src/mod_VelocityTables.f90 FillVelocity raw rules"
    return out


def parse_profiles(path):
    zones = {}
    name = None
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith("VARIABLES"):
                continue
            m = re.match(r'ZONE T="([^"]+)"', line)
            if m:
                name = m.group(1)
                zones[name] = []
                continue
            if line:
                zones[name].append([float(t) for t in line.split()])
    return zones


def namelist_tokens(path):
    """The assignments of a Config.ini's namelist groups as raw value tokens, comments dropped (the
    delivered cases put no '!' inside a string and one assignment on a line)."""
    out, group = {}, None
    with open(path, encoding="utf-8") as f:
        for line in f:
            line = line.split("!")[0].strip()
            if line.startswith("&"):
                group = line[1:].strip().lower()
                out[group] = {}
            elif line == "/":
                group = None
            elif group and "=" in line:
                k, v = line.split("=", 1)
                out[group][k.strip()] = v.split()
    return out


def sha256(path):
    import hashlib
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def parse_sparse(path):
    with open(path) as f:
        header = f.readline().strip().split(",")
        rows = []
        for line in f:
            parts = [p.strip() for p in line.strip().split(",")]
            row = {}
            for k, v in zip(header, parts):
                try:
                    row[k] = float(v)
                except ValueError:
                    row[k] = v
            rows.append(row)
    return rows


def main(ref):
    n1, n2, vel = read_velocity(os.path.join(ref, "cases/low_explicit/velocity_half32_scale2.dat"))
    assert (n1, n2) == (32, 32)
    np.save(os.path.join(HERE, "velocity_half32_scale2.npy"), vel)
    nx0, ny0, gx, gy = read_mesh(os.path.join(ref, "cases/low_explicit/Mesh2d.dat"))
    np.save(os.path.join(HERE, "mesh_8x64.npy"), np.stack([gx, gy]))

    golden = {}
    log = open(os.path.join(ref, "docs/release_checks/low_explicit/stdout.log")).read()
    dt = float(re.search(r"dtPhysical:\s+(\S+)", log).group(1))
    res = [float(t) for t in re.search(r"res:\s+(.*)", log).group(1).split()]
    golden["low_explicit_2step"] = {"dtPhysical": dt, "res": res, "digits": 7,
                                    "source": "docs/release_checks/low_explicit/stdout.log:41-43"}
    for case in ("low_implicit", "high_implicit"):
        golden[case + "_sparse"] = parse_sparse(os.path.join(ref, f"docs/release_checks/{case}/sparse_residual.csv"))
        txt = open(os.path.join(ref, f"docs/release_checks/{case}/stdout.log")).read()
        golden[case + "_summary"] = [l.strip() for l in txt.splitlines() if l.strip().startswith("Implicit iter=")]
    golden["profiles"] = parse_profiles(os.path.join(ref, "docs/couette_results/profiles_three_methods.plt"))
    golden["profiles_columns"] = ["x", "y", "r", "u", "v", "T", "p", "sxx", "sxy", "syy", "qx", "qy"]
    ver = json.load(open(os.path.join(ref, "checks/VERIFICATION.json")))
    golden["static_equilibrium"] = {k: ver[k] for k in ("final_static_le", "static_le_19", "static_le_np1")}
    summ = json.load(open(os.path.join(ref, "docs/couette_results/analysis.json")))["summary"]
    for case in ("low_explicit", "low_implicit", "high_implicit"):
        c = summ[case]
        keep = {k: c[k] for k in ("steps", "status", "selected_final", "c_final") if k in c}
        if "final_walls" in c:
            keep["final_walls"] = {w: {q: c["final_walls"][w][q] for q in ("native_pnn", "native_pnt", "native_qn")}
                                   for w in c["final_walls"]}
        if case == "high_implicit":
            keep["x_spread"] = c["x_spread"]
        keep["source"] = "docs/couette_results/analysis.json summary/" + case
        golden[case + "_final"] = keep
    golden["velocity_tables"] = parse_velocity_tables(os.path.join(ref, "src/mod_VelocityTables.f90"))
    golden["case_namelists"] = {c: namelist_tokens(os.path.join(ref, f"cases/{c}/Config.ini"))
                                for c in ("low_explicit", "low_implicit", "high_implicit")}
    golden["case_file_sha256"] = {f: sha256(os.path.join(ref, "cases/low_implicit", f))
                                  for f in ("Mesh2d.dat", "velocity_half32_scale2.dat")}
    golden["sparse_lines"] = {c: open(os.path.join(ref, f"docs/release_checks/{c}/sparse_residual.csv")).read().splitlines()
                              for c in ("low_implicit", "high_implicit")}
    with open(os.path.join(HERE, "reference_golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
