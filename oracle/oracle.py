"""ctypes binding of the CPU oracle (oracle/awp_oracle.c) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this
module, as the oracle the device results are compared with or as the timed CPU
restatement of the reference.  The product path (cybershake-core_b200/) never
imports it.

PINNING: the reference ships no solver tests or golden outputs and its
Fortran cannot be built here; the oracle is a statement-by-statement
restatement of the Fortran (see the header of awp_oracle.c).  Its set-up stage
is pinned to the reference CUDA variant's host code (setup_reference below),
its time loop to that variant's own velocity and stress kernels run on the
host (tests/golden/make_timeloop_golden.py, within 2e-6 relative L2), and the
synthesis oracle to DirectSynth's own functions (synth_reference).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4", "r5", "r6",
          "lam", "mu", "d1", "qp", "qs"]


class OrcParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dh", C.c_float), ("dt", C.c_float),
        ("nd", C.c_int), ("arbc", C.c_float),
        ("fl", C.c_float), ("fh", C.c_float), ("fp", C.c_float),
        ("socalq", C.c_int), ("nve", C.c_int), ("mediastart", C.c_int), ("nvar", C.c_int),
        ("idyna", C.c_int), ("nst", C.c_int), ("nt", C.c_int), ("ntiskp_sgt", C.c_int),
        ("write_step", C.c_int), ("igreen", C.c_int), ("kinematic", C.c_int), ("rstore", C.c_int),
        ("npc", C.c_int), ("pht", C.c_float),
    ]


# storage formats of r1..r6 the FP32 build emulates (awp_oracle.c ORC_RS_*)
RSTORE = {"f32": 0, "bf16": 1, "bf16_sr": 2, "f16m": 3, "f16m_sr": 4, "bfp6": 5, "bfp33": 6}


_libs = {}


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def load(precision: str = "f32"):
    if precision in _libs:
        return _libs[precision]
    path = os.path.join(_HERE, "liborc_%s.so" % precision)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P, V = C.POINTER, C.c_void_p
    lib.orc_create.restype = V
    lib.orc_create.argtypes = [P(OrcParams)]
    lib.orc_destroy.argtypes = [V]
    lib.orc_set_media.restype = C.c_int
    lib.orc_set_media.argtypes = [V, V]
    lib.orc_set_source.restype = C.c_int
    lib.orc_set_source.argtypes = [V, C.c_int, V, V]
    lib.orc_set_points.restype = C.c_int
    lib.orc_set_points.argtypes = [V, C.c_int, V]
    lib.orc_run.restype = C.c_int
    lib.orc_run.argtypes = [V, C.c_int]
    lib.orc_sgt_file_floats.restype = C.c_int64
    lib.orc_sgt_file_floats.argtypes = [V]
    lib.orc_get_sgt_file.argtypes = [V, V]
    lib.orc_get_chkj.argtypes = [V, V]
    lib.orc_get_field.restype = C.c_int
    lib.orc_get_field.argtypes = [V, C.c_int, V]
    lib.orc_set_field.restype = C.c_int
    lib.orc_set_field.argtypes = [V, C.c_int, V]
    lib.orc_get_extremes.argtypes = [V, V]
    lib.orc_real_bytes.restype = C.c_int
    lib.orc_num_threads.restype = C.c_int
    lib.orc_set_num_threads.argtypes = [C.c_int]
    lib.orc_get_tau.argtypes = [V, V]
    lib.orc_get_sponge.argtypes = [V, V, V, V]
    lib.orc_get_tau12.argtypes = [V, V]
    _libs[precision] = lib
    return lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """One component of the Fortran stepper on the CPU (FP32 or FP64)."""

    def __init__(self, *, nx, ny, nz, dh, dt, nt, nd=20, arbc=0.92, fl=0.01, fh=25.0, fp=0.5,
                 socalq=0, nve=1, mediastart=1, nvar=3, idyna=0, nst=None, ntiskp_sgt=10,
                 write_step=None, igreen=1, precision="f32", threads=0, kinematic=0, rstore="f32", npc=0,
                 pht=0.1):
        self.lib = load(precision)
        if threads:
            self.lib.orc_set_num_threads(threads)
        self.dtype = np.float32 if precision == "f32" else np.float64
        p = OrcParams()
        p.nx, p.ny, p.nz, p.dh, p.dt = nx, ny, nz, dh, dt
        p.nd, p.arbc, p.fl, p.fh, p.fp = nd, arbc, fl, fh, fp
        p.socalq, p.nve, p.mediastart, p.nvar, p.idyna = socalq, nve, mediastart, nvar, idyna
        p.nst = nt if nst is None else nst
        p.nt, p.ntiskp_sgt = nt, ntiskp_sgt
        p.write_step = (nt // ntiskp_sgt) if write_step is None else write_step
        p.igreen = igreen
        p.kinematic = kinematic
        if rstore != "f32" and precision != "f32":
            raise ValueError("r storage formats are emulated by the FP32 build only")
        p.rstore = RSTORE[rstore]
        p.npc, p.pht = npc, pht
        self.p = p
        self.h = self.lib.orc_create(C.byref(p))
        if not self.h:
            raise ValueError("oracle rejected the parameters")

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_media(self, media):
        if media is None:
            st = self.lib.orc_set_media(self.h, None)
        else:
            m = np.ascontiguousarray(media, dtype=np.float32)
            st = self.lib.orc_set_media(self.h, _p(m))
        if st != 0:
            raise ValueError("oracle: bad media")

    def set_source(self, xyz, stf):
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.int32).reshape(-1, 3))
        stf = np.ascontiguousarray(np.asarray(stf, dtype=np.float32).reshape(xyz.shape[0], -1, 6))
        if self.lib.orc_set_source(self.h, xyz.shape[0], _p(xyz), _p(stf)) != 0:
            raise ValueError("oracle: source outside the grid")

    def set_points(self, xyz):
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.int32).reshape(-1, 3))
        if self.lib.orc_set_points(self.h, xyz.shape[0], _p(xyz)) != 0:
            raise ValueError("oracle: point outside the grid")

    def run(self, nsteps):
        return self.lib.orc_run(self.h, nsteps)

    def sgt(self):
        out = np.zeros(int(self.lib.orc_sgt_file_floats(self.h)), dtype=np.float32)
        self.lib.orc_get_sgt_file(self.h, _p(out))
        return out

    def chkj(self):
        out = np.zeros((self.p.nt, 3), dtype=np.float32)
        self.lib.orc_get_chkj(self.h, _p(out))
        return out

    def field(self, name):
        p = self.p
        out = np.zeros((p.nz + 4, p.ny + 4, p.nx + 4), dtype=self.dtype)
        self.lib.orc_get_field(self.h, FIELDS.index(name), _p(out))
        return out

    def set_field(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=self.dtype)
        self.lib.orc_set_field(self.h, FIELDS.index(name), _p(a))

    def extremes(self):
        out = np.zeros(6, dtype=np.float32)
        self.lib.orc_get_extremes(self.h, _p(out))
        return out

    def tau(self):
        """Relaxation times [itz][ity][itx] (relax.f:15-36), set by load_media."""
        out = np.zeros((2, 2, 2), dtype=np.float32)
        self.lib.orc_get_tau(self.h, _p(out))
        return out

    def tau12(self):
        """tau1 and tau2 of viscoop.f:79-88, each [itz][ity][itx] (0-based parities)."""
        out = np.zeros(16, dtype=np.float32)
        self.lib.orc_get_tau12(self.h, _p(out))
        return out[:8].copy(), out[8:].copy()

    def sponge(self):
        """Cerjan factors (cx[nx], cy[ny], cz[nz]), index 0 at the low x / y face
        and at the bottom."""
        p = self.p
        cx, cy, cz = (np.zeros(n, np.float32) for n in (p.nx, p.ny, p.nz))
        self.lib.orc_get_sponge(self.h, _p(cx), _p(cy), _p(cz))
        return cx, cy, cz


def threads():
    return load("f32").orc_num_threads()


def reorder_rwg(sgt: np.ndarray, nt: int, z_source: bool = False) -> np.ndarray:
    """RWG component order of an AWP SGT file image, points x [6][nt]
    (SgtHead/src/reformat_awp.c:39-63, reformat_awp_mpi.c:85-122): XX <- YY,
    YY <- XX, ZZ, XY, XZ <- -YZ, YZ <- -XZ; for the z-force run every value is
    first multiplied by -2.0 in double precision and stored as float."""
    x = np.asarray(sgt, dtype=np.float32).reshape(-1, 6, nt)
    if z_source:
        x = (-2.0 * x.astype(np.float64)).astype(np.float32)
    neg = lambda a: (-1.0 * a.astype(np.float64)).astype(np.float32)
    return np.stack([x[:, 1], x[:, 0], x[:, 2], x[:, 3], neg(x[:, 5]), neg(x[:, 4])], axis=1).reshape(-1)


def rwg_to_awp_media(p: np.ndarray, s: np.ndarray, d: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    """AWP media file order from RWG velocity volumes (SgtHead/src/
    reformat_velocity.c:55-80): input x fastest, then z, then y (km/s, g/cm^3);
    output [z][x][y][vp vs rho], y fastest, each value times 1000.0 (double
    product stored as float)."""
    out = np.empty((nz, nx, ny, 3), dtype=np.float32)
    for v, a in enumerate((p, s, d)):
        a = np.asarray(a, dtype=np.float32).reshape(ny, nz, nx)
        out[..., v] = (a.transpose(1, 2, 0).astype(np.float64) * 1000.0).astype(np.float32)
    return out.reshape(-1)


# ---- reciprocity synthesis (oracle/synth_oracle.c) -------------------------
# Records of the RWG SGT header file and of an SRF point, as
# DirectSynth/src/jbsim/structure.h and srf_structure.h lay them out.
SGTMASTER = np.dtype([("geoproj", "<i4"), ("modellon", "<f4"), ("modellat", "<f4"), ("modelrot", "<f4"),
                      ("xshift", "<f4"), ("yshift", "<f4"), ("globnp", "<i4"), ("localnp", "<i4"), ("nt", "<i4")])
SGTINDEX = np.dtype([("indx", "<i8"), ("xsgt", "<i4"), ("ysgt", "<i4"), ("zsgt", "<i4"), ("h", "<f4")])
SGTHEADER = np.dtype([("indx", "<i8"), ("geoproj", "<i4"), ("modellon", "<f4"), ("modellat", "<f4"),
                      ("modelrot", "<f4"), ("xshift", "<f4"), ("yshift", "<f4"), ("nt", "<i4"), ("xazim", "<f4"),
                      ("dt", "<f4"), ("tst", "<f4"), ("h", "<f4"), ("src_lat", "<f4"), ("src_lon", "<f4"),
                      ("src_dep", "<f4"), ("xsrc", "<i4"), ("ysrc", "<i4"), ("zsrc", "<i4"), ("sgt_lat", "<f4"),
                      ("sgt_lon", "<f4"), ("sgt_dep", "<f4"), ("xsgt", "<i4"), ("ysgt", "<i4"), ("zsgt", "<i4"),
                      ("cdist", "<f4"), ("lam", "<f4"), ("mu", "<f4"), ("rho", "<f4"), ("xmom", "<f4"),
                      ("ymom", "<f4"), ("zmom", "<f4")])
SRFPOINT = np.dtype([("lon", "<f4"), ("lat", "<f4"), ("dep", "<f4"), ("stk", "<f4"), ("dip", "<f4"),
                     ("area", "<f4"), ("tinit", "<f4"), ("dt", "<f4"), ("rake", "<f4"), ("slip1", "<f4"),
                     ("slip2", "<f4"), ("slip3", "<f4"), ("nt1", "<i4"), ("nt2", "<i4"), ("nt3", "<i4"),
                     ("stf1", "<i8"), ("stf2", "<i8"), ("stf3", "<i8")], align=True)

_synth_lib = None


def _load_synth():
    global _synth_lib
    if _synth_lib is None:
        path = os.path.join(_HERE, "liborc_synth.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        V = C.c_void_p
        lib.orc_synth.restype = C.c_int
        lib.orc_synth.argtypes = [V, V, V, C.c_int, V, V, V, C.c_float, C.c_float, C.c_float, C.c_int, C.c_float,
                                  C.c_int, C.c_int, V, V, V, V, C.POINTER(C.c_int)]
        lib.orc_synth_get_indx.restype = None
        lib.orc_synth_get_indx.argtypes = [V, C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(C.c_int64), V]
        _synth_lib = lib
    return _synth_lib


def synth(master, index, headers, comps, slon, slat, dtout, ntout, tstart, variations):
    """Seismograms [nvar][3][ntout] of the rupture variations [(points, pool)]
    for one site, restating DirectSynth's jbsim3d_synth; returns (seis, ntout)."""
    lib = _load_synth()
    m = np.ascontiguousarray(np.asarray(master, SGTMASTER).reshape(1))
    ix = np.ascontiguousarray(index, SGTINDEX)
    hd = np.ascontiguousarray(headers, SGTHEADER)
    cs = [np.ascontiguousarray(c, np.float32) for c in comps]
    ptr = [_p(c) for c in cs] + [None] * (3 - len(cs))
    nv = len(variations)
    npts = len(variations[0][0])
    pts = np.ascontiguousarray(np.concatenate([np.asarray(v[0], SRFPOINT) for v in variations]), SRFPOINT)
    pools = [np.ascontiguousarray(v[1], np.float32) for v in variations]
    off = np.cumsum([0] + [p.size for p in pools[:-1]]).astype(np.int64)
    pool = np.ascontiguousarray(np.concatenate(pools + [np.zeros(1, np.float32)]))
    maxnt, mindt = int(hd[0]["nt"]), np.float32(hd[0]["dt"])
    if np.float32(dtout) < mindt:                     # jbsim3d.c:439-440
        maxnt = int(np.float32(maxnt) * mindt / np.float32(dtout))
    n = 2
    while n < 4 * maxnt:
        n *= 2
    nout = ntout if ntout > 0 else n
    seis = np.zeros((nv, 3, nout), np.float32)
    got = C.c_int()
    rc = lib.orc_synth(_p(m), _p(ix), _p(hd), len(cs), ptr[0], ptr[1], ptr[2], slon, slat, dtout, ntout, tstart,
                       nv, npts, _p(pts), _p(pool), _p(off), _p(seis), C.byref(got))
    if rc:
        raise ValueError("oracle synthesis refused the input (code %d)" % rc)
    assert got.value == nout, (got.value, nout)
    return seis, nout


def synth_get_indx(master, h, lon, lat, dep):
    """(indx, (x, y, z)) of a point in the SGT grid (misc_subs.c:151-173)."""
    lib = _load_synth()
    m = np.ascontiguousarray(np.asarray(master, SGTMASTER).reshape(1))
    indx = C.c_int64()
    xyz = np.zeros(3, np.int32)
    lib.orc_synth_get_indx(_p(m), h, lon, lat, dep, C.byref(indx), _p(xyz))
    return indx.value, tuple(int(v) for v in xyz)


def synth_reference(master, index, headers, comps, slon, slat, dtout, ntout, tstart, variations):
    """The same seismograms from DirectSynth's own functions, built from the
    reference sources into oracle/_ref/libsynth_ref.so (oracle/Makefile.ref);
    None where that library has not been built."""
    path = os.path.join(_HERE, "_ref", "libsynth_ref.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    V = C.c_void_p
    lib.ref_synth.restype = C.c_int
    lib.ref_synth.argtypes = [V, V, V, C.c_int, V, V, V, C.c_float, C.c_float, C.c_float, C.c_int, C.c_float,
                              C.c_int, C.c_int, V, V, V, V, C.POINTER(C.c_int)]
    m = np.ascontiguousarray(np.asarray(master, SGTMASTER).reshape(1))
    ix = np.ascontiguousarray(index, SGTINDEX)
    hd = np.ascontiguousarray(headers, SGTHEADER)
    cs = [np.ascontiguousarray(c, np.float32) for c in comps]
    ptr = [_p(c) for c in cs] + [None] * (3 - len(cs))
    nv, npts = len(variations), len(variations[0][0])
    pts = np.ascontiguousarray(np.concatenate([np.asarray(v[0], SRFPOINT) for v in variations]), SRFPOINT)
    pools = [np.ascontiguousarray(v[1], np.float32) for v in variations]
    off = np.cumsum([0] + [p.size for p in pools[:-1]]).astype(np.int64)
    pool = np.ascontiguousarray(np.concatenate(pools + [np.zeros(1, np.float32)]))
    got = C.c_int()
    n = 1 << 22
    seis = np.zeros(nv * 3 * (ntout if ntout > 0 else n), np.float32)
    rc = lib.ref_synth(_p(m), _p(ix), _p(hd), len(cs), ptr[0], ptr[1], ptr[2], slon, slat, dtout, ntout, tstart, nv,
                       npts, _p(pts), _p(pool), _p(off), _p(seis), C.byref(got))
    if rc:
        raise ValueError("reference synthesis failed (code %d)" % rc)
    return seis[:nv * 3 * got.value].reshape(nv, 3, got.value)


def setup_reference(media, *, nvar=3, nve=1, socalq=0, fp=0.5, fl=0.01, fh=25.0, arbc=0.92, nd=20):
    """The reference CUDA stepper's own host set-up on one rank (AWP-GPU-SGT
    mesh.c inimesh and tausub, cerjan.c inicrj), built from the reference
    sources into oracle/_ref/libsetup_ref.so (oracle/Makefile.ref): media
    [nz][ny][nx][nvar] (z = 0 at the surface) in, a dict of lam mu d1 qp qs in
    the same [z][y][x] order, the extremes (vs, vp, rho min/max), taumin /
    taumax, tau [idx][idy][idz] and the sponge factors out.  None where that
    library has not been built."""
    import tempfile
    path = os.path.join(_HERE, "_ref", "libsetup_ref.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    V, I, F = C.c_void_p, C.c_int, C.c_float
    lib.ref_inimesh.argtypes = [I, I, I, I, I, I, F, F, F, C.c_char_p, V, V, V, V, V, V, V]
    lib.ref_tausub.argtypes = [F, F, V]
    lib.ref_inicrj.argtypes = [F, I, I, I, I, V, V, V]
    m = np.ascontiguousarray(media, np.float32)
    nz, ny, nx = m.shape[:3]
    out = {k: np.zeros((nz, ny, nx), np.float32) for k in ("lam", "mu", "d1", "qp", "qs")}
    ext, tmm, tau8 = np.zeros(6, np.float32), np.zeros(2, np.float32), np.zeros(8, np.float32)
    # mesh.c copies the path into a 40-byte buffer: a short name under /tmp
    fd, fname = tempfile.mkstemp(prefix="m", suffix=".b", dir="/tmp")
    try:
        with os.fdopen(fd, "wb") as f:
            f.write(m.tobytes())
        lib.ref_inimesh(nx, ny, nz, nvar, nve, socalq, fp, fl, fh, fname.encode(), _p(out["lam"]), _p(out["mu"]),
                        _p(out["d1"]), _p(out["qp"]), _p(out["qs"]), _p(ext), _p(tmm))
    finally:
        os.unlink(fname)
    lib.ref_tausub(tmm[0], tmm[1], _p(tau8))
    cx, cy, cz = np.zeros(nx, np.float32), np.zeros(ny, np.float32), np.zeros(nz, np.float32)
    lib.ref_inicrj(arbc, nx, ny, nz, nd, _p(cx), _p(cy), _p(cz))
    out.update(extremes=ext, taumin=tmm[0], taumax=tmm[1], tau=tau8.reshape(2, 2, 2), cx=cx, cy=cy, cz=cz)
    return out
