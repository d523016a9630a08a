"""The reference's case directories, restart files and monitor files (host side).

A reference case directory holds
  Config.ini    the Fortran namelists &config_para and &boundary_para (ReadBaseParameters,
                mod_ImportPara.f90:141-173; defaults Set_default_parameters :53-130);
  Mesh2d.dat    the node coordinates (InitMesh, mod_InitializeFlow.f90:266-330);
  the structured velocity file named by StructuredVelocityFile
                (InitVelocityFromStructuredFile, mod_InitializeFlow.f90:475-509).
`load_case_dir` turns one into a CouetteCase plus its velocity table, with the reference's own
checks and abort codes (201-205 velocity file, 473-474 mesh) raised as `CaseError`.

Restart and monitor files written and read here:
  flow2d.dat, vdf2d.dat, grid2d.grd   write_restart (mod_Output.f90:571-971) and InitFlow_Restart
                                      (mod_InitializeFlow.f90:975-1100), structured branch;
  closed_mass_rank<r>.bin (v4)        WriteMassRestart / ReadMassRestart / RestartIdentity
                                      (mod_ClosedCouetteMass.f90:315-393);
  residual_reference.in               WriteRestartReference (mod_Output.f90:58-76), read back in
                                      mod_R5Observe.f90:176-186;
  sparse_residual.csv                 WriteMonitorRows (mod_R5Observe.f90:322-350);
  ResidualImplicit.plt, the           WriteImplicitResidual (mod_ImplicitDiagnostics.f90:356-399).
  'Implicit iter=' stdout line

Fortran unformatted sequential files are framed as gfortran frames them: every record carries its
byte length as a little-endian int32 before and after the data.  closed_mass_rank<r>.bin is a
stream file (no framing).  Arrays are stored column-major (first index fastest), so the reference's
(i, j, k) array is a C-order [k][j][i] block here.
"""
from dataclasses import dataclass, field
import math
import os
import re
import struct

import numpy as np

from .case import CouetteCase

METHODS = ("Explicit", "ImplicitSteady", "HighOrderImplicit", "S2CN2")
LAP = 2            # halo width of the reference's blocks (mod_Globaldata.f90:95)
MASS_VERSION = 4   # closed_mass_rank*.bin layout version (WriteMassRestart)


class CaseError(ValueError):
    """A case directory or restart file the reference would reject (reference_code: its MPI_Abort
    code where it has one) or that asks for a setting outside this hot path."""

    def __init__(self, msg, reference_code=0):
        super().__init__(msg if not reference_code else f"{msg} (reference abort {reference_code})")
        self.reference_code = reference_code


# ------------------------------------------------------------------------------------------------
# Fortran namelists

class Namelist(dict):
    """One namelist group: lower-case name -> {1-based index: value}."""

    def get(self, key, default=None):
        v = dict.get(self, key.lower())
        if v is None or 1 not in v:
            return default
        return v[1]

    def get_array(self, key, n, default):
        out = list(default)
        for i, x in (dict.get(self, key.lower()) or {}).items():
            if 1 <= i <= n:
                out[i - 1] = x
        return out


_TOKEN = re.compile(r"'(?:[^']|'')*'|\"(?:[^\"]|\"\")*\"|=|,|[^\s,=]+")
_KEY = re.compile(r"^([A-Za-z_][A-Za-z0-9_%]*)(?:\((\d+)(?::(\d+))?\))?$")


def _strip_comment(line):
    quote = None
    for pos, ch in enumerate(line):
        if quote:
            if ch == quote:
                quote = None
        elif ch in "'\"":
            quote = ch
        elif ch == "!":
            return line[:pos]
    return line


def _value(tok):
    if tok[0] in "'\"":
        return tok[1:-1].replace(tok[0] * 2, tok[0])
    low = tok.lower()
    if low in (".true.", ".t.", "t", ".true", "true"):
        return True
    if low in (".false.", ".f.", "f", ".false", "false"):
        return False
    num = low.replace("d", "e")
    if re.fullmatch(r"[+-]?\d+", num):
        return int(num)
    try:
        return float(num)
    except ValueError:
        raise CaseError(f"namelist value '{tok}' is not a number, logical or string") from None


def _group_items(body):
    """Assignments of one group body: [(key, first index, [values])]."""
    toks = _TOKEN.findall(body)
    items = []
    k = 0
    while k < len(toks):
        t = toks[k]
        if t == ",":
            k += 1
            continue
        if k + 1 < len(toks) and toks[k + 1] == "=":
            m = _KEY.match(t)
            if not m:
                raise CaseError(f"bad namelist name '{t}'")
            items.append((m.group(1).lower(), int(m.group(2) or 1), []))
            k += 2
            continue
        if not items:
            raise CaseError(f"namelist value '{t}' before any name")
        rep = re.fullmatch(r"(\d+)\*(.+)", t) if t[0] not in "'\"" else None
        if rep:
            items[-1][2].extend([_value(rep.group(2))] * int(rep.group(1)))
        else:
            items[-1][2].append(_value(t))
        k += 1
    return items


def parse_namelists(text):
    """All &group ... / namelist groups of a file: {group name (lower case): Namelist}.  Text
    outside the groups (comments, the $DIS_para block) is ignored, as READ(nml=) skips it."""
    groups = {}
    name, body = None, []
    for raw in text.splitlines():
        line = _strip_comment(raw).strip()
        if name is None:
            m = re.match(r"^&([A-Za-z_][A-Za-z0-9_]*)\s*(.*)$", line)
            if not m:
                continue
            name, line = m.group(1).lower(), m.group(2)
        # a '/' outside quotes (or &end) closes the group
        quote, end = None, None
        for pos, ch in enumerate(line):
            if quote:
                if ch == quote:
                    quote = None
            elif ch in "'\"":
                quote = ch
            elif ch == "/":
                end = pos
                break
        if end is None and re.search(r"&end\b", line, re.I):
            end = re.search(r"&end\b", line, re.I).start()
        body.append(line if end is None else line[:end])
        if end is not None:
            g = Namelist()
            for key, first, vals in _group_items(" ".join(body)):
                slot = dict.setdefault(g, key, {})
                for off, v in enumerate(vals):
                    slot[first + off] = v
            groups[name] = g
            name, body = None, []
    if name is not None:
        raise CaseError(f"namelist &{name} is not closed")
    return groups


def read_config(path):
    with open(path, encoding="utf-8", errors="replace") as f:
        groups = parse_namelists(f.read())
    for g in ("config_para", "boundary_para"):
        if g not in groups:
            raise CaseError(f"Config.ini has no &{g} namelist ({path})")
    return groups


def _flt(x):
    return f"{x!r}".replace("e", "d") if "e" in f"{x!r}" else f"{x!r}d0"


def _fortran(v):
    if isinstance(v, bool):
        return ".true." if v else ".false."
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, str):
        return "'" + v.replace("'", "''") + "'"
    return _flt(float(v))


def config_text(case, velocity_file="velocity_table.dat", nu=None, nv=None, extra=None):
    """A Config.ini the reference reads as `case` (the keys load_case_dir uses, the rest at the
    values of the reference's delivered cases)."""
    cp = {
        "Iflag_InitFlow": 0, "Ma": 0.0, "Re": 1.0, "AOA": 0.0, "Tinf": case.tinf, "Tw": case.wall_tnative[0],
        "ck": case.ck, "Pr": case.pr, "flag_vislaw": 1, "omega": case.omega, "Tcm": 0.4044,
        "CouetteMuRef": case.mu_ref, "StructuredVelocityFile": velocity_file,
        "TimeIntegration_method": case.method, "UnifiedPhysicalOperators": True, "S2PhysicalGas": 1,
        "S2_mu_ref": case.mu_ref, "S2W1_wall_mode": 1, "S2CartesianMesh": True, "TimeStep_method": 1,
        "CFL": case.cfl, "Implicit_nCFL": case.ncfl, "Implicit_ZhuMovingWall": True,
        "Implicit_InitHaloResync": True, "ClosedCouetteMassRescale": bool(case.mass_rescale),
        "Implicit_MacroSweeps": case.macro_sweeps, "Implicit_MicroSweeps": 1,
        "Implicit_ResidualTol": case.residual_tol, "Implicit_MomentTol": case.moment_tol,
        "Implicit_MinAlpha": case.min_alpha, "Implicit_MaxRetries": 0, "Implicit_MaxIter": case.max_iter,
        "Implicit_ClosedMassConstraint": False, "MAX_ITER": case.max_iter, "Nstep_show": 100,
        "Nstep_write": 100, "Nstep_restart": 100, "Nstep_audit": 0, "Nstep_monitor": 1,
        "Nx_all": case.nx, "Ny_all": case.ny, "NP_X": 1, "NP_Y": case.nslab, "Quadrature_method": 2,
    }
    if case.wall_tnative[1] != case.wall_tnative[0]:
        cp["S2WallTNative"] = list(case.wall_tnative)
    if case.s2w1_time_centered or case.s2w1d_face_time or case.s2w2r_shared_predictor:
        cp["S2W1_time_centered"] = int(case.s2w1_time_centered)
        cp["S2W1D_face_time_consistent"] = int(case.s2w1d_face_time)
        cp["S2W2R_shared_predictor"] = int(case.s2w2r_shared_predictor)
    if nu is not None:
        cp["Nu"], cp["Nv"] = nu, nv
    cp.update(extra or {})
    lines = ["&config_para"]
    for k, v in cp.items():
        vals = v if isinstance(v, (list, tuple)) else [v]
        lines.append(f"{k} = " + " ".join(_fortran(x) for x in vals))
    lines += ["/", "", "&boundary_para", "BC_Type = 10 10 2 2", "BG_geometry = 0", f"FluxWall_type = {case.flux_wall}",
              "ACC = 1.0d0", "CouetteUseW2BWall = .true.",
              "WallUx = 0.0d0 0.0d0 " + " ".join(_flt(float(x)) for x in case.wall_ux), "/", "",
              "$DIS_para", "0", "0", "0", "$DIS_para", ""]
    return "\n".join(lines)


# ------------------------------------------------------------------------------------------------
# Fortran unformatted sequential records

def read_records(path):
    """The records of a gfortran sequential unformatted file, as bytes."""
    with open(path, "rb") as f:
        data = f.read()
    out, off = [], 0
    while off < len(data):
        if off + 4 > len(data):
            raise CaseError(f"{path}: truncated record marker")
        (n,) = struct.unpack_from("<i", data, off)
        if n < 0 or off + 8 + n > len(data):
            raise CaseError(f"{path}: bad record length {n}")
        (n2,) = struct.unpack_from("<i", data, off + 4 + n)
        if n2 != n:
            raise CaseError(f"{path}: record markers {n} / {n2} disagree")
        out.append(data[off + 4: off + 4 + n])
        off += 8 + n
    return out


def write_records(path, records):
    with open(path, "wb") as f:
        for r in records:
            if len(r) > 0x7FFFFFFF - 8:
                raise CaseError(f"{path}: a record of {len(r)} bytes needs gfortran sub-records")
            f.write(struct.pack("<i", len(r)))
            f.write(r)
            f.write(struct.pack("<i", len(r)))


def _i32(*v):
    return struct.pack("<%di" % len(v), *v)


def _f64(a):
    return np.ascontiguousarray(a, dtype="<f8").tobytes()


# ------------------------------------------------------------------------------------------------
# Mesh2d.dat and the velocity file

def read_mesh(path, nx=None, ny=None):
    """Mesh2d.dat -> (gridx, gridy) node arrays [ny+1][nx+1].  Abort 474 when the node counts are
    not (Nx_all+1, Ny_all+1)."""
    recs = read_records(path)
    if len(recs) < 2 or len(recs[0]) < 8:
        raise CaseError(f"{path}: not a Mesh2d.dat file")
    nx0, ny0 = struct.unpack_from("<ii", recs[0])
    if (nx is not None and nx0 != nx + 1) or (ny is not None and ny0 != ny + 1):
        raise CaseError(f"Mesh2d.dat has {nx0} x {ny0} nodes, the case needs {nx + 1} x {ny + 1}", 474)
    vals = np.frombuffer(recs[1], dtype="<f8")
    if vals.size != 2 * nx0 * ny0:
        raise CaseError(f"{path}: coordinate record holds {vals.size} values, expected {2 * nx0 * ny0}", 474)
    return vals[: nx0 * ny0].reshape(ny0, nx0).copy(), vals[nx0 * ny0:].reshape(ny0, nx0).copy()


def write_mesh(path, gridx, gridy):
    ny0, nx0 = gridx.shape
    write_records(path, [_i32(nx0, ny0), _f64(gridx) + _f64(gridy)])


def cartesian_mesh(nx, ny, x_extent=1.0, y_extent=1.0):
    """Uniform node arrays on [0, x_extent] x [0, y_extent] (the delivered cases: the unit square)."""
    i = np.arange(nx + 1, dtype=np.float64)
    j = np.arange(ny + 1, dtype=np.float64)
    gx = np.broadcast_to(i * (x_extent / nx), (ny + 1, nx + 1)).copy()
    gy = np.broadcast_to((j * (y_extent / ny))[:, None], (ny + 1, nx + 1)).copy()
    return gx, gy


def s2_generated_mesh(nx, ny):
    """The mesh InitMesh generates when Mesh2d.dat is absent for an S2 method with S2CartesianMesh and
    S2W1_wall_mode 1 (mod_InitializeFlow.f90:278-290): x = (i-1) 2 pi / Nx_all, y = (j-1) / Ny_all."""
    i = np.arange(nx + 1, dtype=np.float64)
    j = np.arange(ny + 1, dtype=np.float64)
    gx = np.broadcast_to(i * (2.0 * math.acos(-1.0) / nx), (ny + 1, nx + 1)).copy()
    gy = np.broadcast_to((j / ny)[:, None], (ny + 1, nx + 1)).copy()
    return gx, gy


def mesh_spacing(gridx, gridy):
    """(dx, dy) of a uniform Cartesian mesh.  The kernels take one dx and one dy, so the mesh must be
    rectangular (InitializeClosedMass's test, mod_ClosedCouetteMass.f90:216-221, 1e-14) and uniform."""
    ny0, nx0 = gridx.shape
    if np.abs(gridx - gridx[0:1, :]).max() > 1e-14 or np.abs(gridy - gridy[:, 0:1]).max() > 1e-14:
        raise CaseError("mesh is not rectangular Cartesian (requires verified Cartesian Couette geometry)")
    dxs, dys = np.diff(gridx[0]), np.diff(gridy[:, 0])
    dx, dy = float(dxs[0]), float(dys[0])
    if np.abs(dxs - dx).max() > 1e-12 * abs(dx) or np.abs(dys - dy).max() > 1e-12 * abs(dy):
        raise CaseError("mesh is not uniform: this hot path takes one dx and one dy")
    return dx, dy


def cell_centres(gridx, gridy):
    """gridxc_all / gridyc_all (mod_InitializeFlow.f90:300-306): [ny][nx] means of the 4 nodes."""
    xc = 0.25 * (gridx[:-1, :-1] + gridx[:-1, 1:] + gridx[1:, :-1] + gridx[1:, 1:])
    yc = 0.25 * (gridy[:-1, :-1] + gridy[:-1, 1:] + gridy[1:, :-1] + gridy[1:, 1:])
    return xc, yc


def read_velocity_file(path, nu, nv):
    """(u, v, w) of a structured velocity file with the reference's checks: 201 cannot open,
    202 bad size line, 203 sizes differ from (Nu, Nv), 204 bad row, 205 not a tensor-product table
    symmetric about 0 with positive finite weights."""
    try:
        f = open(path)
    except OSError:
        raise CaseError(f"cannot open velocity file {path}", 201) from None
    with f:
        try:
            n1, n2 = (int(t) for t in f.readline().split()[:2])
        except ValueError:
            raise CaseError(f"{path}: bad size line", 202) from None
        if (n1, n2) != (nu, nv):
            raise CaseError(f"{path}: table is {n1} x {n2}, Config.ini says Nu={nu}, Nv={nv}", 203)
        rows = []
        for _ in range(nu * nv):
            parts = f.readline().replace("D", "E").replace("d", "e").split()
            try:
                rows.append([float(t) for t in parts[:3]])
            except ValueError:
                rows = None
            if rows is None or len(rows[-1]) != 3:
                raise CaseError(f"{path}: bad velocity row", 204)
    t = np.array(rows, dtype=np.float64)
    u, v, w = t[:, 0].copy(), t[:, 1].copy(), t[:, 2].copy()
    ok = bool(np.all(np.isfinite(t)) and np.all(w > 0.0))
    i = np.arange(nu)
    for j in range(nv):
        k = i + j * nu
        mirror = (nu - 1 - i) + (nv - 1 - j) * nu
        ok = ok and np.array_equal(u[k], u[i]) and bool(np.all(v[k] == v[j * nu]))
        ok = ok and np.array_equal(u[k], -u[mirror]) and np.array_equal(v[k], -v[mirror])
        ok = ok and np.array_equal(w[k], w[mirror])
    if not ok:
        raise CaseError(f"{path}: not a symmetric tensor-product velocity table", 205)
    return u, v, w


def _es(x, digits=17, width=26, exp_digits=3):
    """Fortran ESw.dEe: one nonzero digit before the point, `digits` after, e-digit exponent."""
    x = float(x)
    if not math.isfinite(x):
        return ("NaN" if math.isnan(x) else ("Infinity" if x > 0 else "-Infinity")).rjust(width)
    s = f"{x:.{digits}E}"
    mant, ex = s.split("E")
    e = int(ex)
    return f"{mant}E{'+' if e >= 0 else '-'}{abs(e):0{exp_digits}d}".rjust(width)


def write_velocity_file(path, u, v, w, nu, nv):
    """The reference's layout: 2I12 sizes, then 3ES26.17E3 rows (u, v, w), k = i + (j-1) Nu."""
    with open(path, "w") as f:
        f.write(f"{nu:12d}{nv:12d}\n")
        for a, b, c in zip(u, v, w):
            f.write(_es(a) + _es(b) + _es(c) + "\n")


# ------------------------------------------------------------------------------------------------
# Case directories

@dataclass
class CaseDir:
    case: CouetteCase
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    gridx: np.ndarray
    gridy: np.ndarray
    config: dict
    run: dict = field(default_factory=dict)   # loop and output controls (MAX_ITER, Nstep_*, Iflag_InitFlow, ...)
    path: str = "."


def _need(cond, what):
    if not cond:
        raise CaseError(f"Config.ini: {what} is outside this hot path")


def case_from_config(groups, mesh=None):
    """CouetteCase of parsed Config.ini namelists (+ mesh node arrays for dx, dy)."""
    c, b = groups["config_para"], groups["boundary_para"]
    method = str(c.get("timeintegration_method", "Explicit")).strip()
    _need(method in METHODS, f"TimeIntegration_method '{method}'")
    implicit = method in ("ImplicitSteady", "HighOrderImplicit")
    s2 = method in ("HighOrderImplicit", "S2CN2")
    nx, ny = int(c.get("nx_all", 0)), int(c.get("ny_all", 0))
    if nx < 1 or ny < 1:
        raise CaseError("Config.ini: Nx_all and Ny_all must be positive")
    npx, npy = int(c.get("np_x", 1)), int(c.get("np_y", 1))
    _need(npx == 1, f"NP_X = {npx} (the device domain keeps the reference's 1 x NP_Y blocking only)")
    if npy < 1 or ny % npy:
        raise CaseError(f"Config.ini: Ny_all = {ny} is not a multiple of NP_Y = {npy}")
    _need(int(c.get("flag_vislaw", 1)) == 1, "flag_vislaw other than the power law (1)")
    _need(bool(c.get("unifiedphysicaloperators", False)), "UnifiedPhysicalOperators = .false.")
    _need(b.get_array("bc_type", 4, [3, 3, 3, 3]) == [10, 10, 2, 2],
          "BC_Type other than 10 10 2 2 (x-periodic, isothermal walls)")
    _need(bool(b.get("couetteusew2bwall", False)), "CouetteUseW2BWall = .false.")
    _need(float(b.get("acc", 1.0)) == 1.0, "ACC other than 1 (fully diffuse walls)")
    if implicit:
        _need(int(c.get("implicit_microsweeps", 1)) == 1, "Implicit_MicroSweeps other than 1")
        _need(int(c.get("implicit_maxretries", 8)) == 0, "Implicit_MaxRetries > 0 (nCFL backoff retries)")
        _need(not bool(c.get("implicit_closedmassconstraint", False)), "Implicit_ClosedMassConstraint")
        _need(bool(c.get("implicit_zhumovingwall", False)), "Implicit_ZhuMovingWall = .false.")
    variant = {"flux_wall": int(b.get("fluxwall_type", 1)),
               "s2w1_time_centered": int(c.get("s2w1_time_centered", 0)),
               "s2w1d_face_time": int(c.get("s2w1d_face_time_consistent", 0)),
               "s2w2r_shared_predictor": int(c.get("s2w2r_shared_predictor", 0))}
    if s2:
        _need(int(c.get("s2w1_wall_mode", 0)) == 1, "S2W1_wall_mode other than 1")
        _need(variant["flux_wall"] in (0, 1), "FluxWall_type other than 0 (kinetic) or 1 (multiscale)")
        fw, tc, fd, sp = (variant[k] for k in ("flux_wall", "s2w1_time_centered", "s2w1d_face_time",
                                               "s2w2r_shared_predictor"))
        if fw == 0 or tc or fd or sp:   # the research wall variants (mod_ImportPara.f90:455-471, :527-528)
            _need(method == "S2CN2" or not (tc or fd or sp),
                  "the W1T / W1D / W2R wall variants on a method other than S2CN2")
            for key, val in (("S2W1_time_centered", tc), ("S2W1D_face_time_consistent", fd),
                             ("S2W2R_shared_predictor", sp)):
                if val not in (0, 1):
                    raise CaseError(f"Config.ini: {key} must be 0 or 1", 200)
            if tc and fw != 0:
                raise CaseError("Config.ini: S2W2 type1 requires centered=0 and face_time_consistent=0", 200)
            if fd and not tc:
                raise CaseError("Config.ini: S2W1D face correction requires W1T midpoint wall", 200)
            if sp and (fw != 1 or int(c.get("ck", 1)) != 1 or float(c.get("pr", 2.0 / 3.0)) != 1.0 or tc or fd
                       or npy != 1):
                raise CaseError("Config.ini: W2R supports only frozen flat type1 BGK setup", 200)
    else:
        variant = {k: 0 for k in variant}
        variant["flux_wall"] = 1
    ck = int(c.get("ck", 1))
    gamma = float(ck + 4) / float(ck + 2)
    mu = float(c.get("couettemuref", -1.0))
    if not mu > 0.0:
        if int(c.get("s2physicalgas", 0)) == 1:
            mu = float(c.get("s2_mu_ref", 0.1))
        else:
            re_ = float(c.get("re", 0.0))
            if re_ == 0.0:
                raise CaseError("Config.ini: no viscosity (CouetteMuRef, S2_mu_ref or Ma / Re)")
            mu = math.sqrt(gamma / 2.0) * float(c.get("ma", 0.0)) / re_
    tw = float(c.get("tw", 0.0))
    theta = c.get_array("s2w1_wall_theta", 2, [None, None])
    native = c.get_array("s2walltnative", 2, [None, None])
    twall = []
    for side in range(2):      # ResolveS2WallTemperatures (mod_ImportPara.f90:274-299)
        tn = tw
        if theta[side] is not None:
            tn = 2.0 * float(theta[side])
        if native[side] is not None:
            tn = float(native[side])
        if not (math.isfinite(tn) and tn > 0.0):
            raise CaseError("effective wall T_native must be positive and finite")
        twall.append(tn)
    wall_ux = b.get_array("wallux", 4, [0.0, 0.0, 0.0, 0.0])
    if mesh is None:
        dx, dy = 1.0 / nx, 1.0 / ny
    else:
        dx, dy = mesh_spacing(*mesh)
    case = CouetteCase(
        nx=nx, ny=ny, dx=dx, dy=dy, ck=ck, pr=float(c.get("pr", 2.0 / 3.0)), omega=float(c.get("omega", 0.5)),
        mu_ref=mu, cfl=float(c.get("cfl", 0.1)), tinf=float(c.get("tinf", 0.0)),
        wall_ux=(float(wall_ux[2]), float(wall_ux[3])), wall_tnative=(twall[0], twall[1]), method=method,
        ncfl=float(c.get("implicit_ncfl", 100.0)), nslab=npy,
        mass_rescale=bool(c.get("closedcouettemassrescale", False)),
        macro_sweeps=int(c.get("implicit_macrosweeps", 2)),
        residual_tol=float(c.get("implicit_residualtol", 1.0e-8)),
        moment_tol=float(c.get("implicit_momenttol", 1.0e-12)),
        min_alpha=float(c.get("implicit_minalpha", 1.0e-6)), max_iter=int(c.get("max_iter", 10000)), **variant)
    if case.mass_rescale and not implicit:
        raise CaseError("ClosedCouetteMassRescale is for the closed-Couette implicit methods only")
    if not (case.tinf > 0.0):
        raise CaseError("Config.ini: Tinf must be positive")
    return case


def load_case_dir(path):
    """A reference case directory -> CaseDir (case, velocity table, mesh, namelists, run controls)."""
    groups = read_config(os.path.join(path, "Config.ini"))
    c = groups["config_para"]
    nx, ny = int(c.get("nx_all", 0)), int(c.get("ny_all", 0))
    method = str(c.get("timeintegration_method", "Explicit")).strip()
    mesh_path = os.path.join(path, "Mesh2d.dat")
    if os.path.exists(mesh_path):
        gx, gy = read_mesh(mesh_path, nx, ny)
    elif bool(c.get("s2cartesianmesh", False)) and method in ("HighOrderImplicit", "S2CN2"):
        gx, gy = s2_generated_mesh(nx, ny)
    else:
        raise CaseError(f"{mesh_path} does not exist", 473)
    case = case_from_config(groups, (gx, gy))
    vfile = str(c.get("structuredvelocityfile", "")).strip()
    nu, nv = int(c.get("nu", 28)), int(c.get("nv", 28))
    if vfile:
        u, v, w = read_velocity_file(os.path.join(path, vfile), nu, nv)
    else:
        _need(method in ("HighOrderImplicit", "S2CN2"), "a velocity set without StructuredVelocityFile")
        table = str(c.get("s2velocitytable", "half32")).strip()
        _need(table in ("half16", "half32"), f"S2VelocityTable '{table}'")
        from .case import velocity_table
        u, v, w = velocity_table(16 if table == "half16" else 32, float(c.get("s2velocityscale", 2.0)))
    run = {k: c.get(k.lower(), d) for k, d in (
        ("Iflag_InitFlow", 0), ("MAX_ITER", 10000), ("Nstep_show", 10), ("Nstep_write", 10000),
        ("Nstep_restart", 100), ("Nstep_monitor", 1), ("Iflag_WriteRestart", 0), ("Implicit_MaxIter", 100000))}
    return CaseDir(case=case, u=u, v=v, w=w, gridx=gx, gridy=gy, config=groups, run=run, path=path)


def write_case_dir(path, case, u, v, w, gridx=None, gridy=None, velocity_file="velocity_table.dat", extra=None):
    """A case directory the reference (and load_case_dir) reads back as `case`."""
    os.makedirs(path, exist_ok=True)
    n = int(round(math.sqrt(len(u))))
    if gridx is None:
        gridx, gridy = cartesian_mesh(case.nx, case.ny, case.dx * case.nx, case.dy * case.ny)
    write_mesh(os.path.join(path, "Mesh2d.dat"), gridx, gridy)
    write_velocity_file(os.path.join(path, velocity_file), u, v, w, n, n)
    with open(os.path.join(path, "Config.ini"), "w") as f:
        f.write(config_text(case, velocity_file, n, n, extra))


# ------------------------------------------------------------------------------------------------
# Restart files (structured branch of write_restart / InitFlow_Restart)

def write_restart(path, W, h, b, nx, ny, gridx=None, gridy=None):
    """flow2d.dat (W), vdf2d.dat (h, b) and, given the mesh, grid2d.grd, from the device layout
    W[ny*nx][4], h/b[ny*nx][nvel] (cell = j nx + i)."""
    nv = h.shape[-1]
    Wc = np.asarray(W, dtype=np.float64).reshape(ny, nx, 4).transpose(2, 0, 1)
    write_records(os.path.join(path, "flow2d.dat"), [_i32(1), _i32(nx, ny, 4), _f64(Wc)])
    hb = np.stack([np.asarray(h, dtype=np.float64).reshape(ny, nx, nv).transpose(2, 0, 1),
                   np.asarray(b, dtype=np.float64).reshape(ny, nx, nv).transpose(2, 0, 1)])
    write_records(os.path.join(path, "vdf2d.dat"), [_i32(1), _i32(nx, ny, 2 * nv), _f64(hb)])
    if gridx is not None:
        xc, yc = cell_centres(gridx, gridy)
        write_records(os.path.join(path, "grid2d.grd"), [_i32(1), _i32(nx, ny), _f64(xc) + _f64(yc)])


def read_restart(path, nx, ny, nv):
    """(W, h, b) in the device layout from flow2d.dat and vdf2d.dat, with InitFlow_Restart's
    conformance checks."""
    recs = read_records(os.path.join(path, "flow2d.dat"))
    if len(recs) < 3 or struct.unpack_from("<iii", recs[1]) != (nx, ny, 4):
        raise CaseError("Restart error: data in flow2d.dat does not conform.")
    Wc = np.frombuffer(recs[2], dtype="<f8")
    if Wc.size != 4 * nx * ny:
        raise CaseError("Restart error: data in flow2d.dat does not conform.")
    W = Wc.reshape(4, ny, nx).transpose(1, 2, 0).reshape(ny * nx, 4).copy()
    recs = read_records(os.path.join(path, "vdf2d.dat"))
    if len(recs) < 3 or struct.unpack_from("<iii", recs[1]) != (nx, ny, 2 * nv):
        raise CaseError("Restart error: data in vdf2d.dat does not conform.")
    hb = np.frombuffer(recs[2], dtype="<f8")
    if hb.size != 2 * nv * nx * ny:
        raise CaseError("Restart error: data in vdf2d.dat does not conform.")
    hb = hb.reshape(2, nv, ny, nx)
    h = hb[0].transpose(1, 2, 0).reshape(ny * nx, nv).copy()
    b = hb[1].transpose(1, 2, 0).reshape(ny * nx, nv).copy()
    return W, h, b


def _seq_sum(x):
    s = 0.0
    for t in np.asarray(x, dtype=np.float64).tolist():
        s += t
    return s


def restart_identity(groups, u, w):
    """RestartIdentity (mod_ClosedCouetteMass.f90:315-322): 31 numbers that bind a mass restart to its
    case.  sum() is sequential, as gfortran evaluates the intrinsic without reassociation."""
    c, b = groups["config_para"], groups["boundary_para"]
    f = float
    ident = [f(c.get("nx_all")), f(c.get("ny_all")), f(c.get("np_x", 1)), f(c.get("np_y", 1)),
             f(c.get("nu", 28)), f(c.get("nv", 28)), f(c.get("cfl", 0.1)), f(c.get("implicit_ncfl", 100.0)),
             f(c.get("ck", 1)), f(c.get("pr", 2.0 / 3.0)), f(c.get("omega", 0.5)), f(c.get("tinf", 0.0)),
             f(c.get("tw", 0.0)), f(c.get("couettemuref", -1.0))]
    ident += [f(x) for x in b.get_array("wallux", 4, [0.0] * 4)]
    ident += [f(x) for x in b.get_array("bc_type", 4, [3] * 4)]
    ident += [f(c.get("flag_vislaw", 1)), f(b.get("fluxwall_type", 1)), f(b.get("acc", 1.0)),
              f(b.get("bg_geometry", 0)), f(c.get("quadrature_method", 1)),
              1.0 if c.get("implicit_zhumovingwall", False) else 0.0,
              1.0 if c.get("implicit_inithaloresync", False) else 0.0]
    u = np.asarray(u, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    ident += [_seq_sum(w), _seq_sum(w * u * u)]
    assert len(ident) == 31
    return np.array(ident, dtype=np.float64)


def _rank_block(field, nx, ny, nslab, rank, ncomp):
    """Rank `rank`'s rows with the LAP halo: x wraps (periodic), seam rows come from the neighbour
    rank, rows beyond a wall are zero (isothermal walls keep no ghost values, mod_Boundary.f90:144)."""
    rows = ny // nslab
    f = np.asarray(field, dtype=np.float64).reshape(ny, nx, ncomp)
    out = np.zeros((rows + 2 * LAP, nx + 2 * LAP, ncomp))
    cols = [(i - LAP) % nx for i in range(nx + 2 * LAP)]
    for jl in range(rows + 2 * LAP):
        j = rank * rows + jl - LAP
        if 0 <= j < ny:
            out[jl] = f[j][cols]
    return out


def write_mass_restart(path, groups, u, w, W, h, b, nx, ny, m0, ledger=(0.0, 0.0, 0.0, 0.0), step=0):
    """closed_mass_rank<r>.bin (version 4) of every rank of the case's 1 x NP_Y blocking."""
    nslab = int(groups["config_para"].get("np_y", 1))
    nv = np.asarray(h).shape[-1]
    ident = restart_identity(groups, u, w)
    rows = ny // nslab
    for r in range(nslab):
        Wr = _rank_block(W, nx, ny, nslab, r, 4)
        hr = _rank_block(h, nx, ny, nslab, r, nv)
        br = _rank_block(b, nx, ny, nslab, r, nv)
        cells = np.concatenate([Wr, hr, br], axis=2)        # per halo cell: conVars, h_vec, b_vec
        with open(os.path.join(path, f"closed_mass_rank{r}.bin"), "wb") as f:
            f.write(_i32(MASS_VERSION, nx, rows, nv, LAP, int(step)))
            f.write(_f64([m0]) + _f64(ledger) + _f64(ident))
            f.write(_f64(cells))


def read_mass_restart(path, groups, u, w, nx, ny, nv, W=None, h=None, b=None):
    """(M0, ledger[4], restart_step) of the closed_mass_rank*.bin set, with ReadMassRestart's checks:
    version, block sizes, the RestartIdentity bit for bit, a valid M0, and (given the flow restart)
    every interior cell equal to it.  The same M0, ledger and step on every rank."""
    nslab = int(groups["config_para"].get("np_y", 1))
    rows = ny // nslab
    ident = restart_identity(groups, u, w)
    seen = None
    ncell = (rows + 2 * LAP) * (nx + 2 * LAP)
    for r in range(nslab):
        fn = os.path.join(path, f"closed_mass_rank{r}.bin")
        try:
            data = open(fn, "rb").read()
        except OSError:
            raise CaseError(f"missing, mismatched, or invalid M0-bearing restart; refusing to redefine M0 ({fn})",
                            941) from None
        hdr = struct.unpack_from("<6i", data, 0)
        m0, = struct.unpack_from("<d", data, 24)
        ledger = np.frombuffer(data, dtype="<f8", count=4, offset=32)
        idf = np.frombuffer(data, dtype="<f8", count=31, offset=64)
        body = np.frombuffer(data, dtype="<f8", offset=64 + 31 * 8)
        ok = hdr[:5] == (MASS_VERSION, nx, rows, nv, LAP) and np.array_equal(idf, ident)
        ok = ok and math.isfinite(m0) and m0 > 0.0 and bool(np.all(np.isfinite(ledger)))
        ok = ok and body.size == ncell * (4 + 2 * nv)
        if ok and W is not None:
            cells = body.reshape(rows + 2 * LAP, nx + 2 * LAP, 4 + 2 * nv)[LAP:LAP + rows, LAP:LAP + nx]
            j0 = r * rows
            Wf = np.asarray(W).reshape(ny, nx, 4)[j0:j0 + rows]
            hf = np.asarray(h).reshape(ny, nx, nv)[j0:j0 + rows]
            bf = np.asarray(b).reshape(ny, nx, nv)[j0:j0 + rows]
            ok = (np.array_equal(cells[..., :4], Wf) and np.array_equal(cells[..., 4:4 + nv], hf)
                  and np.array_equal(cells[..., 4 + nv:], bf))
        if not ok:
            raise CaseError("missing, mismatched, or invalid M0-bearing restart; refusing to redefine M0", 941)
        this = (m0, tuple(ledger.tolist()), hdr[5])
        if seen is not None and this != seen:
            raise CaseError("restart M0, ledger or origin step differs between ranks", 941)
        seen = this
    return seen[0], np.array(seen[1]), seen[2]


# ------------------------------------------------------------------------------------------------
# residual_reference.in and sparse_residual.csv

def write_residual_reference(path, reference_h, reference_b, residual_tol, moment_tol):
    """'(i0,1x,4(es25.16e3,1x))': epoch, reference_h, reference_b, the two tolerances.  An existing
    file's epoch is kept (the original reference epoch survives restarts)."""
    fn = os.path.join(path, "residual_reference.in")
    epoch = 0
    if os.path.exists(fn):
        epoch = read_residual_reference(path)[0]
    vals = (reference_h, reference_b, residual_tol, moment_tol)
    with open(fn, "w") as f:
        f.write(f"{epoch} " + "".join(_es(x, 16, 25) + " " for x in vals) + "\n")


def read_residual_reference(path):
    """(epoch, reference_h, reference_b, residual_tol, moment_tol)."""
    with open(os.path.join(path, "residual_reference.in")) as f:
        t = f.read().replace("D", "E").split()
    try:
        return int(t[0]), float(t[1]), float(t[2]), float(t[3]), float(t[4])
    except (IndexError, ValueError):
        raise CaseError("cannot read residual reference inheritance file") from None


SPARSE_HEADER = ("local_state,cumulative_state,source,original_gate,moment,M_W,M_h,"
                 + ",".join(f"R{k}" for k in range(1, 9)) + ","
                 + ",".join(f"science_{k}" for k in range(1, 23)) + ","
                 + ",".join(f"flux_{k}" for k in range(1, 17))
                 + ",reference_h,reference_b,c_minus_1,mass_rescale_enabled")


def sparse_row(local_state, cumulative_state, report, mass_rescale, source="accepted_convergence_verification"):
    """One sparse_residual.csv line from an implicit report vector (ugks_implicit_steps' report[0..52]
    is the same sequence of values): '(2(i0,","),a,",")' then '(*(es25.16e3,:,","))'."""
    r = np.asarray(report, dtype=np.float64)
    vals = list(r[:52]) + [r[52] if mass_rescale else 0.0, 1.0 if mass_rescale else 0.0]
    return f"{int(local_state)},{int(cumulative_state)},{source}," + ",".join(_es(x, 16, 25) for x in vals)


class SparseResidualWriter:
    """Appends sparse_residual.csv rows, writing the header on the first one."""

    def __init__(self, path, mass_rescale):
        self.fn = os.path.join(path, "sparse_residual.csv")
        self.mass_rescale = mass_rescale

    def append(self, local_state, cumulative_state, report):
        new = not os.path.exists(self.fn)
        with open(self.fn, "a") as f:
            if new:
                f.write(SPARSE_HEADER + "\n")
            f.write(sparse_row(local_state, cumulative_state, report, self.mass_rescale) + "\n")


# ------------------------------------------------------------------------------------------------
# ResidualImplicit.plt and the implicit stdout line (WriteImplicitResidual,
# mod_ImplicitDiagnostics.f90:356-399).  Both print the science of the pre-update evaluation
# (SciencePack, mod_R5Observe.f90:27-32: the view of the accepted state is restored away before
# they are written) with the moment error of the update (after the rescale, the accepted state's).

RESIDUAL_IMPLICIT_HEADER = (
    "VARIABLES = iter dtPhysicalMin nCFL alpha rhoResidual rhoUResidual rhoVResidual energyResidual "
    "hResidual bResidual momentError massDefect retries wallTime prSeconds lusgsSeconds "
    "correctionExchangeSeconds evolutionSeconds retryTotal rhoRelative rhoURelative rhoVRelative "
    "energyRelative rhoAbsolute rhoUAbsolute rhoVAbsolute energyAbsolute hRelative bRelative hAbsolute "
    "bAbsolute microForwardSeconds microBackwardSeconds microForwardBackwardExchangeSeconds c_minus_1 "
    "mass_rescale_enabled")

PRE_SCIENCE = 57   # report[57..78]: science_1..22 of the pre-update evaluation


def _fe(x, width, digits):
    """Fortran 1PEw.d: d.ddd, then E+dd (E dropped for a 3-digit exponent)."""
    x = float(x)
    if not math.isfinite(x):
        return ("NaN" if math.isnan(x) else ("Infinity" if x > 0 else "-Infinity")).rjust(width)
    mant, ex = f"{x:.{digits}E}".split("E")
    e = int(ex)
    tail = f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) <= 99 else f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    return (mant + tail).rjust(width)


def _implicit_values(report, ncfl):
    r = np.asarray(report, dtype=np.float64)
    sci = r[PRE_SCIENCE:PRE_SCIENCE + 22]
    return r, sci, {"dt": r[55], "ncfl": ncfl, "alpha": r[53], "moment": r[1], "mass": sci[19]}


def residual_implicit_row(it, report, ncfl, mass_rescale, wall_time=0.0):
    """One ResidualImplicit.plt row: '(I12,1P,11E18.9,I8,5E18.9,I12,15E18.9,2ES25.16E3)'.  The
    reference's phase timers (PR, LU-SGS, exchange, evolution, micro sweeps) are written as 0: the
    device pseudo-step is one graph launch and is timed only as a whole (wall_time)."""
    r, sci, v = _implicit_values(report, ncfl)
    a = [v["dt"], v["ncfl"], v["alpha"], *sci[0:4], sci[12], sci[13], v["moment"], v["mass"]]
    b = [wall_time, 0.0, 0.0, 0.0, 0.0]
    c = [*sci[4:8], *sci[8:12], sci[14], sci[15], sci[16], sci[17], 0.0, 0.0, 0.0]
    return (f"{int(it):12d}" + "".join(_fe(x, 18, 9) for x in a) + f"{0:8d}" + "".join(_fe(x, 18, 9) for x in b)
            + f"{0:12d}" + "".join(_fe(x, 18, 9) for x in c)
            + _es(r[52] if mass_rescale else 0.0, 16, 25) + _es(1.0 if mass_rescale else 0.0, 16, 25))


def implicit_stdout_line(it, report, ncfl, wall_time=0.0):
    """The 'Implicit iter=...' line: '(A,I0,1P,11(A,E12.4),2(A,I0))'."""
    r, sci, v = _implicit_values(report, ncfl)
    names = (("nCFL", v["ncfl"]), ("alpha", v["alpha"]), ("Rrho", sci[0]), ("RrhoU", sci[1]), ("RrhoV", sci[2]),
             ("RE", sci[3]), ("Rh", sci[12]), ("Rb", sci[13]), ("moment", v["moment"]), ("mass", v["mass"]),
             ("wall", wall_time))
    return f"Implicit iter={int(it)}" + "".join(f" {k}={_fe(x, 12, 4)}" for k, x in names) + " retries=0 retryTotal=0"


class ResidualImplicitWriter:
    """ResidualImplicit.plt: replaced by the first row of a run, appended afterwards."""

    def __init__(self, path, ncfl, mass_rescale):
        self.fn = os.path.join(path, "ResidualImplicit.plt")
        self.ncfl, self.mass_rescale = ncfl, mass_rescale
        self.started = False

    def append(self, it, report, wall_time):
        with open(self.fn, "a" if self.started else "w") as f:
            if not self.started:
                f.write(RESIDUAL_IMPLICIT_HEADER + "\n")
            f.write(residual_implicit_row(it, report, self.ncfl, self.mass_rescale, wall_time) + "\n")
        self.started = True
