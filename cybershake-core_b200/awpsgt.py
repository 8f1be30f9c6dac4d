"""ctypes binding of libawpsgt, the B200 AWP-ODC-SGT stepper (include/awp_sgt.h).

Host-side mirror of the reference's interface for the strain-Green-tensor run:
the same parameters as IN3D (AWP-ODC-SGT/src/io.f:327-417), the same input
layouts (media [z][y][x][nvar] with z = 0 at the surface, source [nst][6],
cordfile points) and the same raw SGT file image (pmcl3d.f:1589-1601).

The library is the compiled CUDA path; there is no CPU fallback.  Importing this
module on a machine without the built library raises ImportError, and creating
a solver without a usable GPU returns AWP_ERR_CUDA as an exception.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libawpsgt.so")
WRITE_HEAD_PATH = os.path.join(_HERE, "lib", "write_head")
REFORMAT_AWP_PATH = os.path.join(_HERE, "lib", "reformat_awp")
REFORMAT_VELOCITY_PATH = os.path.join(_HERE, "lib", "reformat_velocity")
PMCL3D_PATH = os.path.join(_HERE, "lib", "pmcl3d")

AWP_OK = 0
STATUS = {0: "AWP_OK", 1: "AWP_ERR_IO", 2: "AWP_ERR_PARAM", 3: "AWP_ERR_OOM", 4: "AWP_ERR_CUDA",
          5: "AWP_ERR_UNSTABLE", 6: "AWP_ERR_TIMEOUT", 7: "AWP_ERR_STATE", 8: "AWP_ERR_BUSY",
          9: "AWP_ERR_CANCELLED"}
PREC = {"f32": 0, "bf16": 1, "f16": 2, "mixed": 3, "bfp": 4}
KERNEL = {"auto": 0, "two_sweep": 1, "fused": 2, "staged": 3, "staged_fma": 4}
FIELDS = ["u1", "v1", "w1", "xx", "yy", "zz", "xy", "xz", "yz", "r1", "r2", "r3", "r4", "r5", "r6",
          "lam", "mu", "d1", "qp", "qs"]

# Every symbol include/awp_sgt.h declares.
EXPORTED = [
    "awp_params_default", "awp_create", "awp_load_media", "awp_load_media_file", "awp_set_source",
    "awp_set_points", "awp_run", "awp_sgt_file_floats", "awp_get_sgt", "awp_get_chkj", "awp_get_field",
    "awp_get_stats", "awp_reset", "awp_destroy", "awp_footprint_bytes", "awp_bytes_per_cell_update",
    "awp_status_string", "awp_last_error", "awp_read_in3d", "awp_parse_command_line",
    "awp_params_from_in3d", "awp_read_source", "awp_read_cordfile", "awp_free", "awp_profile_steps",
    "awp_run_async", "awp_query", "awp_sync", "awp_device_field", "awp_field_energy", "awp_energy",
    "awp_server_create", "awp_submit", "awp_poll", "awp_cancel", "awp_wait", "awp_server_time",
    "awp_server_destroy", "awp_sgt_floats_for", "awp_field_energy_noalloc", "awp_server_configure",
    "awp_get_sgt_rwg", "awp_sgt_reorder_rwg", "awp_write_sgt_header", "awp_load_media_rwg",
    "awp_reformat_velocity", "awp_get_tuning", "awp_set_tuning", "awp_autotune", "awp_release_cached_memory",
    "awp_set_field", "awp_checkpoint_write", "awp_checkpoint_read", "awp_device_memory", "awp_get_plane",
]
# Every symbol include/awp_synth.h declares.
EXPORTED_SYNTH = [
    "awp_synth_create", "awp_synth_destroy", "awp_synth_set_sgt", "awp_synth_load_sgt_files",
    "awp_synth_add_variation", "awp_synth_add_variation_borrowed", "awp_synth_add_srf_file", "awp_synth_clear_variations", "awp_synth_run",
    "awp_synth_seismograms", "awp_synth_write_grm", "awp_synth_get_info", "awp_srf_read",
]


class Layout(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("pitch", C.c_int), ("plane", C.c_int),
                ("vol", C.c_int64)]


class AwpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dh", C.c_float), ("dt", C.c_float),
        ("nt", C.c_int), ("nd", C.c_int), ("arbc", C.c_float),
        ("fl", C.c_float), ("fh", C.c_float), ("fp", C.c_float),
        ("socalq", C.c_int), ("nve", C.c_int), ("mediastart", C.c_int), ("nvar", C.c_int),
        ("idyna", C.c_int), ("nst", C.c_int), ("ntiskp_sgt", C.c_int), ("write_step", C.c_int),
        ("ncomp", C.c_int), ("igreen", C.c_int * 3), ("precision", C.c_int), ("kernel", C.c_int),
        ("device", C.c_int), ("monitor_every", C.c_int), ("kinematic", C.c_int),
        ("npc", C.c_int), ("pht", C.c_float),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("steps_done", C.c_int64), ("seconds_loop", C.c_double), ("gcell_updates_per_s", C.c_double),
        ("bytes_per_cell_update", C.c_double), ("device_bytes", C.c_double),
        ("vp_min", C.c_float), ("vp_max", C.c_float), ("vs_min", C.c_float), ("vs_max", C.c_float),
        ("rho_min", C.c_float), ("rho_max", C.c_float), ("energy", C.c_double),
    ]


class Tuning(C.Structure):
    """awp_tuning: launch shapes of the steppers (results do not depend on them)."""
    _fields_ = [(n, C.c_int) for n in ("kchunk_staged", "staged_qslow", "staged_rpt", "staged_rpt_vel", "unroll",
                                        "ty", "kchunk", "kchunk_sweep", "staged_batch", "sm_limit")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class KernelTimes(C.Structure):
    _fields_ = [("nkernels", C.c_int), ("name", (C.c_char * 32) * 8), ("launches", C.c_int * 8),
                ("ms_per_launch", C.c_double * 8), ("bytes_per_launch", C.c_double * 8)]

    def as_dict(self):
        return {self.name[k].value.decode(): {"launches": self.launches[k], "ms": self.ms_per_launch[k],
                                              "bytes": self.bytes_per_launch[k]}
                for k in range(self.nkernels)}


_S = C.c_char * 512


class In3dC(C.Structure):
    """awp_in3d: everything IN3D carries (AWP-ODC-SGT/src/io.f:327-417)."""
    _fields_ = (
        [("igreen", C.c_int), ("tmax", C.c_float), ("dh", C.c_float), ("dt", C.c_float),
         ("npc", C.c_int), ("nd", C.c_int), ("arbc", C.c_float), ("pht", C.c_float)]
        + [(n, C.c_int) for n in ("nsrc", "nst", "nx", "ny", "nz", "npx", "npy", "npz",
                                   "ifault", "checkpoint", "isfcvlm", "imd5", "ivelocity", "mediarestart",
                                   "nvar", "iost", "partdeg", "io_opt", "iperf", "idyna", "socalq", "nve")]
        + [(n, C.c_float) for n in ("mu_s", "mu_d", "fl", "fh", "fp")]
        + [(n, C.c_int) for n in ("read_step", "write_step", "write_step2",
                                   "nbgx", "nedx", "nskpx", "nbgy", "nedy", "nskpy", "nbgz", "nedz", "nskpz",
                                   "ntiskp", "nbgx2", "nedx2", "nskpx2", "nbgy2", "nedy2", "nskpy2",
                                   "nbgz2", "nedz2", "nskpz2", "ntiskp2", "ntiskp_sgt")]
        + [(n, _S) for n in ("chkp", "chkj", "insrc", "invel", "insgt", "sxgro", "sygro", "szgro",
                              "sxgro2", "sygro2", "szgro2", "sgtgro", "sgsn", "out_dir")]
        + [("gpu_cli", C.c_int), ("nt", C.c_int)]
    )


_lib = None


class SgtHeadArgs(C.Structure):
    """awp_sgthead_args: the arguments of SgtHead's write_head."""
    _fields_ = [("modelbox", C.c_char_p), ("coordfile", C.c_char_p), ("fdloc", C.c_char_p),
                ("gridout", C.c_char_p), ("spacing", C.c_float), ("nt", C.c_int), ("dt", C.c_float),
                ("sgt_tinc", C.c_int), ("component", C.c_char_p), ("moment", C.c_float), ("flo", C.c_float),
                ("media_file", C.c_char_p), ("mu_corr", C.c_int)]


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


def write_sgt_header(outfile: str, modelbox: str, coordfile: str, fdloc: str, gridout: str, spacing: float,
                     nt: int, dt: float, sgt_tinc: int, component: str, moment: float, flo: float,
                     media_file: str, mu_corr: bool = False) -> None:
    """awp_write_sgt_header: the .sgthead file of one SGT component."""
    a = SgtHeadArgs(modelbox.encode(), coordfile.encode(), fdloc.encode(), gridout.encode(), spacing, nt, dt,
                    sgt_tinc, component.encode(), moment, flo, media_file.encode(), int(bool(mu_corr)))
    _check(load_library().awp_write_sgt_header(C.byref(a), outfile.encode()))


def read_sgt_header(path: str):
    """(sgtmaster, sgtindex[np], sgtheader[np]) records of a header file."""
    raw = np.fromfile(path, dtype=np.uint8)
    m = raw[:SGTMASTER.itemsize].view(SGTMASTER)[0]
    npts = int(m["globnp"])
    o = SGTMASTER.itemsize
    ix = raw[o:o + npts * SGTINDEX.itemsize].view(SGTINDEX)
    o += npts * SGTINDEX.itemsize
    hd = raw[o:o + npts * SGTHEADER.itemsize].view(SGTHEADER)
    return m, ix, hd


def sgt_reorder_rwg(sgt: np.ndarray, nt: int, z_source: bool = False) -> np.ndarray:
    """awp_sgt_reorder_rwg on a host SGT file image (points x [6][nt])."""
    a = np.ascontiguousarray(sgt, dtype=np.float32)
    npts = a.size // (6 * nt)
    out = np.empty(npts * 6 * nt, dtype=np.float32)
    _check(load_library().awp_sgt_reorder_rwg(_ptr(a), npts, nt, int(bool(z_source)), _ptr(out)))
    return out


class SynthParams(C.Structure):
    """awp_synth_params."""
    _fields_ = [("device", C.c_int), ("slon", C.c_float), ("slat", C.c_float), ("dtout", C.c_float),
                ("ntout", C.c_int), ("tstart", C.c_float), ("rv_batch", C.c_int)]


class SynthInfo(C.Structure):
    """awp_synth_info."""
    _fields_ = [("ntout", C.c_int), ("ntsum", C.c_int), ("nsgt_points", C.c_int), ("non_exact", C.c_int),
                ("nvariations", C.c_int), ("ncomp", C.c_int), ("terms", C.c_int64), ("macs", C.c_int64),
                ("seconds_plan", C.c_double), ("seconds_device", C.c_double), ("seconds_conv", C.c_double),
                ("gpu_launches", C.c_int), ("seconds_gf", C.c_double)]


# awp_srf_point (jbsim/srf_structure.h srf_apointvalues with pool offsets)
SRFPOINT = np.dtype([("lon", "<f4"), ("lat", "<f4"), ("dep", "<f4"), ("stk", "<f4"), ("dip", "<f4"),
                     ("area", "<f4"), ("tinit", "<f4"), ("dt", "<f4"), ("rake", "<f4"), ("slip1", "<f4"),
                     ("slip2", "<f4"), ("slip3", "<f4"), ("nt1", "<i4"), ("nt2", "<i4"), ("nt3", "<i4"),
                     ("stf1", "<i8"), ("stf2", "<i8"), ("stf3", "<i8")], align=True)
# awp_seisheader (DirectSynth/src/jbsim/structure.h seisheader, 56 bytes)
SEISHEADER = np.dtype([("version", "S8"), ("site_name", "S8"), ("padding", "S8"), ("source_id", "<i4"),
                       ("rupture_id", "<i4"), ("rup_var_id", "<i4"), ("dt", "<f4"), ("nt", "<i4"),
                       ("comps", "<i4"), ("det_max_freq", "<f4"), ("stoch_max_freq", "<f4")])


def read_srf(path: str, binary: bool = False):
    """awp_srf_read: (points as SRFPOINT records, slip-rate sample pool)."""
    lib = load_library()
    pts = C.c_void_p()
    pool = C.c_void_p()
    n = C.c_int()
    npool = C.c_int64()
    _check(lib.awp_srf_read(path.encode(), int(bool(binary)), C.byref(pts), C.byref(n), C.byref(pool),
                            C.byref(npool)))
    try:
        a = np.frombuffer((C.c_char * (n.value * SRFPOINT.itemsize)).from_address(pts.value), SRFPOINT).copy() \
            if n.value else np.zeros(0, SRFPOINT)
        b = np.frombuffer((C.c_float * npool.value).from_address(pool.value), np.float32).copy() \
            if npool.value else np.zeros(0, np.float32)
    finally:
        lib.awp_free(pts)
        lib.awp_free(pool)
    return a, b


class Synth:
    """Reciprocity seismogram synthesis for one site and one rupture: the
    DirectSynth worker step (jbsim3d_synth) with the SGT set held on the GPU."""

    def __init__(self, slon: float, slat: float, dtout: float, ntout: int = -1, tstart: float = 0.0,
                 device: int = 0, rv_batch: int = 0):
        self.lib = load_library()
        self.p = SynthParams(device, slon, slat, dtout, ntout, tstart, rv_batch)
        h = C.c_void_p()
        _check(self.lib.awp_synth_create(C.byref(self.p), C.byref(h)))
        self.h = h
        self.nvar = 0
        self._borrowed = []          # arrays the library reads in place until run / clear

    def close(self):
        if getattr(self, "h", None):
            self.lib.awp_synth_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_sgt(self, master, index, headers, comps: Sequence[np.ndarray]):
        """SGT set from host arrays: the x component's records and 1-3
        [globnp][6][nt] float32 arrays (x, y, z)."""
        m = np.ascontiguousarray(np.asarray(master, SGTMASTER).reshape(1))
        ix = np.ascontiguousarray(index, SGTINDEX)
        hd = np.ascontiguousarray(headers, SGTHEADER)
        cs = [np.ascontiguousarray(c, np.float32) for c in comps]
        ptrs = [_ptr(c) if i < len(cs) else None for i, c in enumerate(cs + [None] * (3 - len(cs)))]
        _check(self.lib.awp_synth_set_sgt(self.h, _ptr(m), _ptr(ix), _ptr(hd), len(cs), *ptrs))

    def load_sgt_files(self, xhead: str, xdata: str, yhead: Optional[str] = None, ydata: Optional[str] = None,
                       zhead: Optional[str] = None, zdata: Optional[str] = None):
        enc = lambda x: x.encode() if x else None
        _check(self.lib.awp_synth_load_sgt_files(self.h, enc(xhead), enc(xdata), enc(yhead), enc(ydata),
                                                 enc(zhead), enc(zdata)))

    def add_variation(self, rup_var_id: int, points: np.ndarray, pool: np.ndarray, borrow: bool = False):
        """Adds a variation; with borrow the library reads the arrays in place
        (this object keeps them alive until the next run / clear)."""
        pts = np.ascontiguousarray(points, SRFPOINT)
        pl = np.ascontiguousarray(pool, np.float32)
        fn = self.lib.awp_synth_add_variation_borrowed if borrow else self.lib.awp_synth_add_variation
        _check(fn(self.h, rup_var_id, _ptr(pts), len(pts), _ptr(pl), pl.size))
        if borrow:
            self._borrowed.append((pts, pl))
        self.nvar += 1

    def add_srf_file(self, rup_var_id: int, path: str, binary: bool = False):
        _check(self.lib.awp_synth_add_srf_file(self.h, rup_var_id, path.encode(), int(bool(binary))))
        self.nvar += 1

    def clear_variations(self):
        _check(self.lib.awp_synth_clear_variations(self.h))
        self.nvar = 0
        self._borrowed = []

    def run(self) -> np.ndarray:
        """Synthesises every variation; returns [nvar][3][ntout] (vertical, north, east)."""
        _check(self.lib.awp_synth_run(self.h))
        return self.seismograms()

    def info(self) -> SynthInfo:
        i = SynthInfo()
        _check(self.lib.awp_synth_get_info(self.h, C.byref(i)))
        return i

    def seismograms(self) -> np.ndarray:
        i = self.info()
        out = np.empty((i.nvariations, 3, i.ntout), np.float32)
        _check(self.lib.awp_synth_seismograms(self.h, _ptr(out), out.size))
        return out

    def write_grm(self, path: str, site: str = "", source_id: int = 0, rupture_id: int = 0,
                  det_max_freq: float = 0.0, stoch_max_freq: float = 0.0, version: str = "12.10"):
        h = np.zeros(1, SEISHEADER)
        h["version"], h["site_name"] = version.encode(), site.encode()[:7]
        h["source_id"], h["rupture_id"] = source_id, rupture_id
        h["det_max_freq"], h["stoch_max_freq"] = det_max_freq, stoch_max_freq
        _check(self.lib.awp_synth_write_grm(self.h, path.encode(), _ptr(h)))


def read_grm(path: str, ncomp_out: int, ntout: int):
    """Records of a merged seismogram file: (headers, samples[nvar][ncomp_out][ntout])."""
    raw = np.fromfile(path, np.uint8)
    rec = SEISHEADER.itemsize + 4 * ncomp_out * ntout
    n = raw.size // rec
    hd = np.stack([raw[i * rec:i * rec + SEISHEADER.itemsize].view(SEISHEADER)[0] for i in range(n)]) \
        if n else np.zeros(0, SEISHEADER)
    data = np.stack([raw[i * rec + SEISHEADER.itemsize:(i + 1) * rec].view(np.float32).reshape(ncomp_out, ntout)
                     for i in range(n)]) if n else np.zeros((0, ncomp_out, ntout), np.float32)
    return hd, data


def load_library(path: str = LIB_PATH):
    """Loads libawpsgt.so; raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libawpsgt not built: {path} missing (run __graft_entry__.build())")
    lib = C.CDLL(path)
    P = C.POINTER
    sig = {
        "awp_params_default": (None, [P(Params)]),
        "awp_create": (C.c_int, [P(Params), P(C.c_void_p)]),
        "awp_load_media": (C.c_int, [C.c_void_p, C.c_void_p]),
        "awp_load_media_file": (C.c_int, [C.c_void_p, C.c_char_p]),
        "awp_set_source": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
        "awp_set_points": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
        "awp_run": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
        "awp_sgt_file_floats": (C.c_int64, [C.c_void_p]),
        "awp_get_sgt": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
        "awp_get_chkj": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
        "awp_get_field": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
        "awp_get_plane": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
        "awp_set_field": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
        "awp_device_memory": (C.c_int, [C.c_int, P(C.c_int64), P(C.c_int64)]),
        "awp_checkpoint_write": (C.c_int, [C.c_void_p, C.c_char_p]),
        "awp_checkpoint_read": (C.c_int, [C.c_void_p, C.c_char_p, P(C.c_int)]),
        "awp_get_stats": (C.c_int, [C.c_void_p, P(Stats)]),
        "awp_reset": (C.c_int, [C.c_void_p]),
        "awp_destroy": (C.c_int, [C.c_void_p]),
        "awp_footprint_bytes": (C.c_int64, [P(Params), C.c_int]),
        "awp_bytes_per_cell_update": (C.c_double, [P(Params)]),
        "awp_status_string": (C.c_char_p, [C.c_int]),
        "awp_last_error": (C.c_char_p, []),
        "awp_read_in3d": (C.c_int, [C.c_char_p, P(In3dC)]),
        "awp_parse_command_line": (C.c_int, [C.c_int, P(C.c_char_p), P(In3dC)]),
        "awp_params_from_in3d": (None, [P(In3dC), P(Params)]),
        "awp_read_source": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
        "awp_read_cordfile": (C.c_int, [C.c_char_p, P(C.c_int), P(P(C.c_int))]),
        "awp_free": (None, [C.c_void_p]),
        "awp_profile_steps": (C.c_int, [C.c_void_p, C.c_int, P(KernelTimes)]),
        "awp_run_async": (C.c_int, [C.c_void_p, C.c_int]),
        "awp_query": (C.c_int, [C.c_void_p]),
        "awp_sync": (C.c_int, [C.c_void_p]),
        "awp_device_field": (C.c_int, [C.c_void_p, C.c_int, C.c_int, P(C.c_void_p), P(Layout)]),
        "awp_field_energy": (C.c_int, [P(C.c_void_p), C.c_int, P(Layout), C.c_void_p]),
        "awp_field_energy_noalloc": (C.c_int, [P(C.c_void_p), C.c_int, P(Layout), C.c_void_p, C.c_void_p]),
        "awp_energy": (C.c_int, [C.c_void_p, C.c_void_p]),
        "awp_server_create": (C.c_int, [C.c_int, C.c_int64, C.c_int, C.c_int, P(C.c_void_p)]),
        "awp_submit": (C.c_int, [C.c_void_p, C.c_void_p, P(C.c_int64)]),
        "awp_poll": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p]),
        "awp_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
        "awp_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_void_p]),
        "awp_server_time": (C.c_double, [C.c_void_p]),
        "awp_server_destroy": (C.c_int, [C.c_void_p]),
        "awp_server_configure": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double]),
        "awp_get_sgt_rwg": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
        "awp_sgt_reorder_rwg": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p]),
        "awp_write_sgt_header": (C.c_int, [P(SgtHeadArgs), C.c_char_p]),
        "awp_load_media_rwg": (C.c_int, [C.c_void_p, C.c_char_p]),
        "awp_reformat_velocity": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_char_p]),
        "awp_sgt_floats_for": (C.c_int64, [P(Params), C.c_int]),
        "awp_release_cached_memory": (None, []),
        "awp_get_tuning": (C.c_int, [C.c_void_p, P(Tuning)]),
        "awp_set_tuning": (C.c_int, [C.c_void_p, P(Tuning)]),
        "awp_autotune": (C.c_int, [P(Params), C.c_void_p, C.c_int, C.c_char_p, P(Tuning), P(C.c_double)]),
        "awp_synth_create": (C.c_int, [P(SynthParams), P(C.c_void_p)]),
        "awp_synth_destroy": (None, [C.c_void_p]),
        "awp_synth_set_sgt": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_void_p]),
        "awp_synth_load_sgt_files": (C.c_int, [C.c_void_p] + [C.c_char_p] * 6),
        "awp_synth_add_variation": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int64]),
        "awp_synth_add_variation_borrowed": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                                       C.c_int64]),
        "awp_synth_add_srf_file": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_int]),
        "awp_synth_clear_variations": (C.c_int, [C.c_void_p]),
        "awp_synth_run": (C.c_int, [C.c_void_p]),
        "awp_synth_seismograms": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
        "awp_synth_write_grm": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p]),
        "awp_synth_get_info": (C.c_int, [C.c_void_p, P(SynthInfo)]),
        "awp_srf_read": (C.c_int, [C.c_char_p, C.c_int, P(C.c_void_p), P(C.c_int), P(C.c_void_p), P(C.c_int64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(st: int):
    if st != AWP_OK:
        raise AwpError(st, load_library().awp_last_error().decode())


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def make_params(nx, ny, nz, dh, dt, nt, *, nd=20, arbc=0.92, fl=0.01, fh=25.0, fp=0.5, socalq=0, nve=1,
                mediastart=1, nvar=3, idyna=0, nst=None, ntiskp_sgt=10, write_step=None,
                igreen: Sequence[int] = (1,), precision="f32", kernel="auto", device=0,
                monitor_every=0, kinematic=0, npc=0, pht=0.1) -> Params:
    lib = load_library()
    p = Params()
    lib.awp_params_default(C.byref(p))
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dh, p.dt, p.nt = dh, dt, nt
    p.nd, p.arbc = nd, arbc
    p.fl, p.fh, p.fp = fl, fh, fp
    p.socalq, p.nve, p.mediastart, p.nvar, p.idyna = socalq, nve, mediastart, nvar, idyna
    p.nst = nt if nst is None else nst
    p.ntiskp_sgt = ntiskp_sgt
    p.write_step = (nt // ntiskp_sgt) if write_step is None else write_step
    p.ncomp = len(igreen)
    for q, g in enumerate(igreen):
        p.igreen[q] = g
    p.precision = PREC[precision] if isinstance(precision, str) else precision
    p.kernel = KERNEL[kernel] if isinstance(kernel, str) else kernel
    p.device = device
    p.monitor_every = monitor_every
    p.kinematic = kinematic
    p.npc, p.pht = npc, pht
    return p


def nt_file(p: Params) -> int:
    """Samples per component in the raw SGT file (pmcl3d.f:1590-1594)."""
    return ((p.nt // p.write_step) * p.write_step) // p.ntiskp_sgt


class Solver:
    """One SGT solve (1-3 components sharing one medium) on one GPU."""

    def __init__(self, params: Params):
        self.lib = load_library()
        self.p = params
        h = C.c_void_p()
        _check(self.lib.awp_create(C.byref(params), C.byref(h)))
        self.h = h
        self.npts = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.awp_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_media(self, media: Optional[np.ndarray]):
        if media is None:
            _check(self.lib.awp_load_media(self.h, None))
            return
        m = np.ascontiguousarray(media, dtype=np.float32)
        _check(self.lib.awp_load_media(self.h, _ptr(m)))

    def load_media_file(self, path: str):
        _check(self.lib.awp_load_media_file(self.h, path.encode()))

    def set_source(self, comp: int, xyz, stf: np.ndarray):
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.int32).reshape(-1, 3))
        stf = np.ascontiguousarray(np.asarray(stf, dtype=np.float32).reshape(xyz.shape[0], -1, 6))
        _check(self.lib.awp_set_source(self.h, comp, xyz.shape[0], _ptr(xyz), _ptr(stf)))

    def set_points(self, xyz):
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.int32).reshape(-1, 3))
        self.npts = xyz.shape[0]
        _check(self.lib.awp_set_points(self.h, xyz.shape[0], _ptr(xyz)))

    def run(self, nsteps: int, with_sgt: bool = False):
        if with_sgt:
            out = np.zeros((self.p.ncomp, self.sgt_file_floats()), dtype=np.float32)
            _check(self.lib.awp_run(self.h, nsteps, _ptr(out)))
            return out
        _check(self.lib.awp_run(self.h, nsteps, None))
        return None

    def reset(self):
        _check(self.lib.awp_reset(self.h))

    def sgt_file_floats(self) -> int:
        return int(self.lib.awp_sgt_file_floats(self.h))

    def sgt(self, comp: int = 0) -> np.ndarray:
        out = np.zeros(self.sgt_file_floats(), dtype=np.float32)
        _check(self.lib.awp_get_sgt(self.h, comp, _ptr(out)))
        return out

    def load_media_rwg(self, prefix: str):
        """Media from RWG volumes prefix.p / .s / .d (awp_load_media_rwg)."""
        _check(self.lib.awp_load_media_rwg(self.h, prefix.encode()))

    def sgt_rwg(self, comp: int = 0, z_source: bool = False) -> np.ndarray:
        """SGT file image of one component in RWG order (awp_get_sgt_rwg)."""
        out = np.empty(max(int(self.lib.awp_sgt_file_floats(self.h)), 0), dtype=np.float32)
        _check(self.lib.awp_get_sgt_rwg(self.h, comp, int(bool(z_source)), _ptr(out)))
        return out

    def chkj(self, comp: int = 0) -> np.ndarray:
        out = np.zeros((self.p.nt, 3), dtype=np.float32)
        _check(self.lib.awp_get_chkj(self.h, comp, _ptr(out)))
        return out

    def field(self, name: str, comp: int = 0) -> np.ndarray:
        p = self.p
        out = np.zeros((p.nz + 4, p.ny + 4, p.nx + 4), dtype=np.float32)
        _check(self.lib.awp_get_field(self.h, comp, FIELDS.index(name), _ptr(out)))
        return out

    def plane(self, name: str, k: int, comp: int = 0) -> np.ndarray:
        """awp_get_plane: the interior [ny][nx] of level k (1..nz, nz = the
        free surface) of a wavefield or stress."""
        p = self.p
        out = np.zeros((p.ny, p.nx), dtype=np.float32)
        _check(self.lib.awp_get_plane(self.h, comp, FIELDS.index(name), k, _ptr(out)))
        return out

    def set_field(self, name: str, arr, comp: int = 0) -> None:
        """awp_set_field: one state field from the padded host layout
        [nz+4][ny+4][nx+4] float32."""
        p = self.p
        a = np.ascontiguousarray(arr, dtype=np.float32)
        if a.shape != (p.nz + 4, p.ny + 4, p.nx + 4):
            raise ValueError("set_field: shape %s, expected %s" % (a.shape, (p.nz + 4, p.ny + 4, p.nx + 4)))
        _check(self.lib.awp_set_field(self.h, comp, FIELDS.index(name), _ptr(a)))

    def checkpoint_write(self, directory: str) -> None:
        """awp_checkpoint_write: the reference's checkpoint files in `directory`."""
        _check(self.lib.awp_checkpoint_write(self.h, directory.encode()))

    def checkpoint_read(self, directory: str) -> int:
        """awp_checkpoint_read: restores the newest checkpoint; returns its step
        (0 when none was found)."""
        t = C.c_int(0)
        _check(self.lib.awp_checkpoint_read(self.h, directory.encode(), C.byref(t)))
        return t.value

    def run_async(self, nsteps: int):
        _check(self.lib.awp_run_async(self.h, nsteps))

    def query(self) -> bool:
        r = self.lib.awp_query(self.h)
        if r < 0:
            raise AwpError(4, self.lib.awp_last_error().decode())
        return bool(r)

    def sync(self):
        _check(self.lib.awp_sync(self.h))

    def energy(self) -> np.ndarray:
        out = np.zeros(self.p.ncomp, dtype=np.float64)
        _check(self.lib.awp_energy(self.h, _ptr(out)))
        return out

    def device_field(self, name: str, comp: int = 0):
        """(device pointer, Layout) of a field of the current wavefield."""
        ptr = C.c_void_p()
        L = Layout()
        _check(self.lib.awp_device_field(self.h, comp, FIELDS.index(name), C.byref(ptr), C.byref(L)))
        return ptr.value, L

    def profile(self, nsteps: int) -> dict:
        """Advances nsteps steps with CUDA events around every kernel launch."""
        kt = KernelTimes()
        _check(self.lib.awp_profile_steps(self.h, nsteps, C.byref(kt)))
        return kt.as_dict()

    def stats(self) -> Stats:
        s = Stats()
        _check(self.lib.awp_get_stats(self.h, C.byref(s)))
        return s

    def tuning(self) -> Tuning:
        t = Tuning()
        _check(self.lib.awp_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, t: Tuning):
        _check(self.lib.awp_set_tuning(self.h, C.byref(t)))


def device_memory(device: int = 0):
    """awp_device_memory: (bytes held by live solvers, bytes idle in the cache)."""
    live, idle = C.c_int64(0), C.c_int64(0)
    _check(load_library().awp_device_memory(device, C.byref(live), C.byref(idle)))
    return live.value, idle.value


def release_cached_memory():
    """Returns the device blocks kept from destroyed solvers to the driver."""
    load_library().awp_release_cached_memory()


def autotune(params: Params, media: Optional[np.ndarray] = None, trial_steps: int = 20,
             cache: Optional[str] = None):
    """Times candidate launch shapes on the grid and settings of `params` and
    returns (best Tuning, Gcell-updates/s).  media as for Solver.load_media, or
    None for a homogeneous medium; with `cache` the result is read from / kept in
    that file, keyed by grid, components, precision, stepper and GPU model."""
    lib = load_library()
    t = Tuning()
    rate = C.c_double()
    m = None
    if media is not None:
        m = np.ascontiguousarray(media, dtype=np.float32)
    _check(lib.awp_autotune(C.byref(params), None if m is None else _ptr(m), trial_steps,
                            None if cache is None else cache.encode(), C.byref(t), C.byref(rate)))
    return t, rate.value


class Request(C.Structure):
    _fields_ = [("params", Params), ("media", C.c_void_p), ("nsrc", C.c_int * 3), ("src_xyz", C.c_void_p * 3),
                ("stf", C.c_void_p * 3), ("npts", C.c_int), ("pts", C.c_void_p), ("sgt_out", C.c_void_p)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("steps_done", C.c_int64), ("footprint", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


REQ_STATE = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


class Server:
    """Continuous-batching SGT server on one GPU (awp_server_* in the C ABI)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, max_active: int = 4, chunk_steps: int = 100):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib.awp_server_create(device, hbm_budget, max_active, chunk_steps, C.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, params: Params, media: Optional[np.ndarray], sources, points) -> int:
        """sources: per component a (xyz [nsrc][3], stf [nsrc][nst][6]) pair."""
        rq = Request()
        rq.params = params
        keep = []
        if media is not None:
            m = np.ascontiguousarray(media, dtype=np.float32)
            keep.append(m)
            rq.media = m.ctypes.data
        for q, (xyz, stf) in enumerate(sources):
            xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
            stf = np.ascontiguousarray(np.asarray(stf, np.float32).reshape(xyz.shape[0], -1, 6))
            keep += [xyz, stf]
            rq.nsrc[q] = xyz.shape[0]
            rq.src_xyz[q] = xyz.ctypes.data
            rq.stf[q] = stf.ctypes.data
        pts = np.ascontiguousarray(np.asarray(points, np.int32).reshape(-1, 3))
        keep.append(pts)
        rq.npts = pts.shape[0]
        rq.pts = pts.ctypes.data
        nf = int(self.lib.awp_sgt_floats_for(C.byref(params), rq.npts))
        out = np.zeros((params.ncomp, max(nf, 1)), dtype=np.float32)
        keep.append(out)
        rq.sgt_out = out.ctypes.data
        rid = C.c_int64()
        _check(self.lib.awp_submit(self.h, C.byref(rq), C.byref(rid)))
        self._keep[rid.value] = (keep, out)
        return rid.value

    def configure(self, policy: str = "fifo", fill_cells: float = 0.0, chunk_cells: float = 0.0):
        """Admission order ("fifo", "sjf" or "fifo_srpt": arrival order with a
        double SM share for the resident solve with the least remaining work),
        GPU-fill threshold and chunk size in cell-updates (<= 0 keeps the
        current value)."""
        _check(self.lib.awp_server_configure(self.h, {"fifo": 0, "sjf": 1, "fifo_srpt": 2}[policy], fill_cells, chunk_cells))

    def poll(self, rid: int) -> dict:
        info = RequestInfo()
        _check(self.lib.awp_poll(self.h, rid, C.byref(info)))
        return info.as_dict()

    def wait(self, rid: int, timeout: float = 3600.0):
        info = RequestInfo()
        _check(self.lib.awp_wait(self.h, rid, timeout, C.byref(info)))
        return info.as_dict(), self._keep[rid][1]

    def cancel(self, rid: int):
        _check(self.lib.awp_cancel(self.h, rid))

    def time(self) -> float:
        return float(self.lib.awp_server_time(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.awp_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def field_energy(ptrs: Sequence[int], layout: Layout, ncomp: int) -> np.ndarray:
    """awp_field_energy on device arrays (u,v,w per component); the result is
    written to a device buffer and copied back through torch."""
    import torch
    arr = (C.c_void_p * len(ptrs))(*ptrs)
    out = torch.zeros(ncomp, dtype=torch.float64, device="cuda")
    _check(load_library().awp_field_energy(arr, ncomp, C.byref(layout), C.c_void_p(out.data_ptr())))
    return out.cpu().numpy()


def field_energy_noalloc(ptrs: Sequence[int], layout: Layout, ncomp: int, out, stream: int = 0) -> None:
    """awp_field_energy_noalloc: enqueues the energy of the device arrays into
    the caller's device buffer `out` (a torch float64 tensor of >= ncomp
    elements) on `stream` (a raw cudaStream_t handle) and returns at once.
    The library looks up its scratch on the current device, so `out` must
    live there."""
    import torch
    if not (isinstance(out, torch.Tensor) and out.is_cuda and out.dtype == torch.float64):
        raise ValueError("field_energy_noalloc: out must be a CUDA float64 tensor")
    if out.device.index != torch.cuda.current_device():
        raise ValueError("field_energy_noalloc: out is on cuda:%d, the current device is cuda:%d"
                         % (out.device.index, torch.cuda.current_device()))
    if ncomp < 1 or out.numel() < ncomp or len(ptrs) < 3 * ncomp:
        raise ValueError("field_energy_noalloc: %d components need 3*%d field pointers and %d outputs "
                         "(got %d and %d)" % (ncomp, ncomp, ncomp, len(ptrs), out.numel()))
    arr = (C.c_void_p * len(ptrs))(*ptrs)
    _check(load_library().awp_field_energy_noalloc(arr, ncomp, C.byref(layout), C.c_void_p(out.data_ptr()),
                                                   C.c_void_p(stream)))


def read_in3d(path: str) -> In3dC:
    o = In3dC()
    _check(load_library().awp_read_in3d(path.encode(), C.byref(o)))
    return o


def parse_command_line(argv: Sequence[str]) -> In3dC:
    """Parses a pmcl3d command line (argv[0] is the program name)."""
    arr = (C.c_char_p * len(argv))(*[a.encode() for a in argv])
    o = In3dC()
    _check(load_library().awp_parse_command_line(len(argv), arr, C.byref(o)))
    return o


def params_from_in3d(o: In3dC) -> Params:
    p = Params()
    load_library().awp_params_from_in3d(C.byref(o), C.byref(p))
    return p


def read_source(path: str, ifault: int, nsrc: int, nst: int):
    xyz = np.zeros((nsrc, 3), dtype=np.int32)
    stf = np.zeros((nsrc, nst, 6), dtype=np.float32)
    _check(load_library().awp_read_source(path.encode(), ifault, nsrc, nst, _ptr(xyz), _ptr(stf)))
    return xyz, stf


def read_cordfile(path: str) -> np.ndarray:
    lib = load_library()
    n = C.c_int()
    ptr = C.POINTER(C.c_int)()
    _check(lib.awp_read_cordfile(path.encode(), C.byref(n), C.byref(ptr)))
    out = np.ctypeslib.as_array(ptr, shape=(n.value * 3,)).copy().reshape(-1, 3) if n.value else np.zeros((0, 3), np.int32)
    lib.awp_free(ptr)
    return out


def footprint_bytes(p: Params, npts: int) -> int:
    return int(load_library().awp_footprint_bytes(C.byref(p), npts))


def bytes_per_cell_update(p: Params) -> float:
    return float(load_library().awp_bytes_per_cell_update(C.byref(p)))
