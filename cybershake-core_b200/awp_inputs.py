"""Seeded synthetic inputs in the reference formats, and their file writers.

No public dataset is involved: the benchmark configurations use media, source
time functions and SGT point sets generated here from fixed seeds.

  media      float32 [z][y][x][nvar], z = 0 at the free surface
             (record layout read by AWP-ODC-SGT/src/structure.f:142-173)
  source     text: "x y z" then NST lines "axx, ayy, azz, axz, ayz, axy"
             (AWP-ODC-SGT/src/source.f:170-198, AWP-*-SGT/utils/build_src.py)
  cordfile   count, then "x y z" lines sorted by (y, x, z)
             (AWP-ODC-SGT/src/io.f:424-434, SgtHead/gen_awp_cordfile.py:35-39)
  IN3D       "value NAME" lines in the order of AWP-ODC-SGT/src/io.f:327-417

Random numbers come from splitmix64 so that any other language can reproduce
the point sets bit for bit.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014), the published 64-bit mixer."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def below(self, n: int) -> int:
        """Uniform integer in [0, n) by rejection (no modulo bias)."""
        limit = (1 << 64) - ((1 << 64) % n)
        while True:
            v = self.next_u64()
            if v < limit:
                return v % n


def sgt_points(nx: int, ny: int, zmax: int, npts: int, seed: int = 0) -> np.ndarray:
    """npts distinct cordfile points, x in [1,nx], y in [1,ny], z in [1,zmax]
    (z = 1 at the surface), sorted by (y, x, z) like gen_awp_cordfile.py."""
    if npts > nx * ny * zmax:
        raise ValueError("more points than cells")
    rng = SplitMix64(seed)
    seen = set()
    pts: List[Tuple[int, int, int]] = []
    while len(pts) < npts:
        x = 1 + rng.below(nx)
        y = 1 + rng.below(ny)
        z = 1 + rng.below(zmax)
        if (x, y, z) in seen:
            continue
        seen.add((x, y, z))
        pts.append((x, y, z))
    pts.sort(key=lambda p: (p[1], p[0], p[2]))
    return np.asarray(pts, dtype=np.int32)


def gaussian_derivative_stf(nst: int, dt: float, f0: float = 0.5, amp: float = 1.0e15,
                            column: int = 0) -> np.ndarray:
    """[nst][6] source table; column `column` holds
    amp * (t - t0) * exp(-(pi f0 (t - t0))^2), t = n*dt, t0 = 1.5/f0 (FP64)."""
    t = np.arange(nst, dtype=np.float64) * dt
    t0 = 1.5 / f0
    s = amp * (t - t0) * np.exp(-(math.pi * f0 * (t - t0)) ** 2)
    out = np.zeros((nst, 6), dtype=np.float32)
    out[:, column] = s.astype(np.float32)
    return out


def homogeneous_media(nx: int, ny: int, nz: int, vp: float = 6000.0, vs: float = 3464.0,
                      rho: float = 2700.0) -> np.ndarray:
    m = np.empty((nz, ny, nx, 3), dtype=np.float32)
    m[..., 0] = vp
    m[..., 1] = vs
    m[..., 2] = rho
    return m


def correlated_field(shape: Tuple[int, int, int], corr_cells: float, seed: int) -> np.ndarray:
    """Zero-mean, unit-std Gaussian random field with Gaussian autocorrelation
    exp(-r^2/a^2), a = corr_cells (white noise filtered by a Gaussian of
    sigma a/2).  Built on a grid coarsened so the filter spans about 4 coarse
    cells, then trilinearly interpolated; shape is (nz, ny, nx)."""
    sigma = corr_cells / 2.0
    cf = max(1, int(sigma // 2))
    cshape = tuple(int(math.ceil(n / cf)) + 2 for n in shape)
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(cshape).astype(np.float32)
    s = sigma / cf
    spec = np.fft.rfftn(w)
    kz = np.fft.fftfreq(cshape[0])[:, None, None]
    ky = np.fft.fftfreq(cshape[1])[None, :, None]
    kx = np.fft.rfftfreq(cshape[2])[None, None, :]
    g = np.exp(-2.0 * (math.pi * s) ** 2 * (kx * kx + ky * ky + kz * kz))
    f = np.fft.irfftn(spec * g, s=cshape, axes=(0, 1, 2)).astype(np.float32)
    f -= f.mean()
    f /= max(float(f.std()), 1e-30)
    if cf == 1:
        return np.ascontiguousarray(f[1:1 + shape[0], 1:1 + shape[1], 1:1 + shape[2]])
    out = f
    for ax, n in enumerate(shape):
        pos = np.arange(n, dtype=np.float64) / cf + 0.5
        i0 = np.floor(pos).astype(np.int64)
        wgt = (pos - i0).astype(np.float32)
        a = np.take(out, i0, axis=ax)
        b = np.take(out, i0 + 1, axis=ax)
        bshape = [1, 1, 1]
        bshape[ax] = n
        wgt = wgt.reshape(bshape)
        out = a * (1 - wgt) + b * wgt
    out -= out.mean()
    out /= max(float(out.std()), 1e-30)
    return np.ascontiguousarray(out.astype(np.float32))


def _field_slab(coarse: np.ndarray, cf: int, shape, z0: int, z1: int) -> np.ndarray:
    """Planes z0..z1-1 of the trilinear interpolation of a coarse field (the
    interpolation of correlated_field, before normalisation)."""
    out = coarse
    sl = [(z0, z1), (0, shape[1]), (0, shape[2])]
    for ax in range(3):
        lo, hi = sl[ax]
        pos = np.arange(lo, hi, dtype=np.float64) / cf + 0.5
        i0 = np.floor(pos).astype(np.int64)
        wgt = (pos - i0).astype(np.float32)
        a = np.take(out, i0, axis=ax)
        b = np.take(out, i0 + 1, axis=ax)
        bshape = [1, 1, 1]
        bshape[ax] = hi - lo
        wgt = wgt.reshape(bshape)
        out = a * (1 - wgt) + b * wgt
    return out.astype(np.float32)


def _layered_media_slabs(nx, ny, nz, dh, seed, nlayers, vs_top, vs_bot, pert_std, corr_len, basin, slab=16):
    """layered_media for grids too large to hold several full-size temporaries:
    the same recipe evaluated z-slab by z-slab (the correlated field is
    normalised with statistics gathered over all slabs first)."""
    depth = (np.arange(nz, dtype=np.float64) + 0.5) * dh
    thick = nz * dh / nlayers
    layer = np.minimum((depth // thick).astype(np.int64), nlayers - 1)
    vs_l = vs_top * (vs_bot / vs_top) ** (np.arange(nlayers) / max(nlayers - 1, 1))
    shape = (nz, ny, nx)
    coarse, cf = None, 1
    mean, std = 0.0, 1.0
    if pert_std > 0:
        sigma = (corr_len / dh) / 2.0
        cf = max(1, int(sigma // 2))
        cshape = tuple(int(math.ceil(n / cf)) + 2 for n in shape)
        rng = np.random.default_rng(seed)
        w = rng.standard_normal(cshape).astype(np.float32)
        sc = sigma / cf
        kz = np.fft.fftfreq(cshape[0])[:, None, None]
        ky = np.fft.fftfreq(cshape[1])[None, :, None]
        kx = np.fft.rfftfreq(cshape[2])[None, None, :]
        g = np.exp(-2.0 * (math.pi * sc) ** 2 * (kx * kx + ky * ky + kz * kz))
        coarse = np.fft.irfftn(np.fft.rfftn(w) * g, s=cshape, axes=(0, 1, 2)).astype(np.float32)
        coarse -= coarse.mean()
        coarse /= max(float(coarse.std()), 1e-30)
        s1 = s2 = 0.0
        for z0 in range(0, nz, slab):
            f = _field_slab(coarse, cf, shape, z0, min(nz, z0 + slab)).astype(np.float64)
            s1 += float(f.sum())
            s2 += float((f * f).sum())
        n = float(nx) * ny * nz
        mean = s1 / n
        std = max(math.sqrt(max(s2 / n - mean * mean, 0.0)), 1e-30)
    if basin is not None:
        x = (np.arange(nx) + 0.5) * dh
        y = (np.arange(ny) + 0.5) * dh
        r2 = ((x[None, :] - basin["cx"]) / basin["rx"]) ** 2 + ((y[:, None] - basin["cy"]) / basin["ry"]) ** 2
        floor = basin["depth"] * np.sqrt(np.clip(1.0 - r2, 0.0, None))
    m = np.empty((nz, ny, nx, 3), dtype=np.float32)
    for z0 in range(0, nz, slab):
        z1 = min(nz, z0 + slab)
        vs = np.empty((z1 - z0, ny, nx), dtype=np.float32)
        for k in range(z0, z1):
            vs[k - z0] = np.float32(vs_l[layer[k]])
            if basin is not None:
                inside = depth[k] < floor
                if inside.any():
                    frac = np.where(inside, depth[k] / np.maximum(floor, 1e-9), 1.0)
                    vsb = (400.0 + 600.0 * frac).astype(np.float32)
                    vs[k - z0] = np.where(inside, np.minimum(vs[k - z0], vsb), vs[k - z0])
        if coarse is not None:
            pert = ((_field_slab(coarse, cf, shape, z0, z1) - mean) / std).astype(np.float32)
            vs *= (1.0 + pert_std * pert).astype(np.float32)
        vp = (1.73 * vs).astype(np.float32)
        m[z0:z1, ..., 0] = vp
        m[z0:z1, ..., 1] = vs
        m[z0:z1, ..., 2] = (310.0 * np.power(vp.astype(np.float64), 0.25)).astype(np.float32)
    return m


def layered_media(nx: int, ny: int, nz: int, dh: float, seed: int, nlayers: int = 8,
                  vs_top: float = 500.0, vs_bot: float = 4000.0, pert_std: float = 0.05,
                  corr_len: float = 2000.0,
                  basin: Optional[dict] = None) -> np.ndarray:
    """1-D layered model (nlayers of equal thickness, Vs geometric from vs_top to
    vs_bot), Vp = 1.73 Vs, rho = 310 Vp^0.25 (Gardner, SI units), times
    (1 + pert_std * correlated field) on Vp and Vs.  Optional basin: ellipsoid
    {cx, cy, rx, ry, depth} (metres) where Vs ramps from 400 m/s at the surface
    to 1000 m/s at its floor.  Grids above 2e8 cells are built z-slab by
    z-slab (same recipe, bounded host memory)."""
    if float(nx) * ny * nz > 2.0e8:
        return _layered_media_slabs(nx, ny, nz, dh, seed, nlayers, vs_top, vs_bot, pert_std, corr_len, basin)
    depth = (np.arange(nz, dtype=np.float64) + 0.5) * dh
    thick = nz * dh / nlayers
    layer = np.minimum((depth // thick).astype(np.int64), nlayers - 1)
    vs_l = vs_top * (vs_bot / vs_top) ** (np.arange(nlayers) / max(nlayers - 1, 1))
    vs1 = vs_l[layer].astype(np.float32)
    vs = np.broadcast_to(vs1[:, None, None], (nz, ny, nx)).astype(np.float32)
    if basin is not None:
        x = (np.arange(nx) + 0.5) * dh
        y = (np.arange(ny) + 0.5) * dh
        r2 = ((x[None, :] - basin["cx"]) / basin["rx"]) ** 2 + ((y[:, None] - basin["cy"]) / basin["ry"]) ** 2
        floor = basin["depth"] * np.sqrt(np.clip(1.0 - r2, 0.0, None))        # (ny, nx)
        for k in range(nz):
            inside = depth[k] < floor
            if not inside.any():
                continue
            frac = np.where(inside, depth[k] / np.maximum(floor, 1e-9), 1.0)
            vsb = (400.0 + 600.0 * frac).astype(np.float32)
            vs[k] = np.where(inside, np.minimum(vs[k], vsb), vs[k])
    if pert_std > 0:
        pert = correlated_field((nz, ny, nx), corr_len / dh, seed)
        scale = (1.0 + pert_std * pert).astype(np.float32)
    else:
        scale = np.ones((nz, ny, nx), dtype=np.float32)
    vs = vs * scale
    vp = (1.73 * vs).astype(np.float32)
    rho = (310.0 * np.power(vp.astype(np.float64), 0.25)).astype(np.float32)
    m = np.empty((nz, ny, nx, 3), dtype=np.float32)
    m[..., 0] = vp
    m[..., 1] = vs
    m[..., 2] = rho
    return m


def stable_dt(media: np.ndarray, dh: float, courant: float = 0.45) -> float:
    """Time step from the CFL number vp_max*dt/dh (the CHKP stability number)."""
    return float(courant * dh / float(media[..., 0].max()))


# ---------------------------------------------------------------------------
# writers
# ---------------------------------------------------------------------------

def write_media(path: str, media: np.ndarray):
    np.ascontiguousarray(media, dtype=np.float32).tofile(path)


def write_source_text(path: str, xyz: Sequence[int], stf: np.ndarray):
    with open(path, "w") as f:
        f.write("%d %d %d\n" % tuple(int(v) for v in xyz))
        for row in np.asarray(stf, dtype=np.float32):
            f.write(", ".join("%.9e" % float(v) for v in row) + "\n")


def write_source_binary(path: str, xyz: Sequence[int], stf: np.ndarray):
    with open(path, "wb") as f:
        np.asarray(xyz, dtype=np.int32).tofile(f)
        np.asarray(stf, dtype=np.float32).tofile(f)


def write_cordfile(path: str, pts: np.ndarray, comment: Optional[str] = None):
    with open(path, "w") as f:
        if comment:
            f.write("# %s\n" % comment)
        f.write("%d\n" % len(pts))
        for x, y, z in pts:
            f.write("%d %d %d\n" % (x, y, z))


@dataclass
class In3d:
    """IN3D values (io.f:327-417 order); defaults follow AWP-ODC-SGT/utils/data/IN3D.ref."""
    igreen: int = 1
    tmax: float = 10.0
    dh: float = 200.0
    dt: float = 0.01
    npc: int = 0
    nd: int = 20
    arbc: float = 0.92
    pht: float = 0.1
    nsrc: int = 1
    nst: int = 1000
    nx: int = 160
    ny: int = 160
    nz: int = 80
    npx: int = 1
    npy: int = 1
    npz: int = 1
    ifault: int = 0
    checkpoint: int = 0
    isfcvlm: int = 0
    imd5: int = 0
    ivelocity: int = 1
    mediarestart: int = 1
    nvar: int = 3
    iost: int = 1
    partdeg: int = 1
    io_opt: int = 1
    perf_meas: int = 1
    idyna: int = 0
    socalq: int = 1
    nve: int = 1
    mu_s: float = 0.677
    mu_d: float = 0.525
    fl: float = 0.01
    fh: float = 25.0
    fp: float = 0.5
    read_step: int = 1000
    write_step: int = 100
    write_step2: int = 100
    rec: Tuple[int, ...] = (1, 160, 10, 1, 160, 10, 1, 80, 10)
    ntiskp: int = 100000
    rec2: Tuple[int, ...] = (1, 160, 10, 1, 160, 10, 1, 80, 10)
    ntiskp2: int = 1000000
    ntiskp_sgt: int = 10
    chkp: str = "output_ckp/CHKP"
    chkj: str = "output_ckp/CHKJ"
    insrc: str = "input/src"
    invel: str = "input/media"
    insgt: str = "input/cordfile"
    sxgro: str = "output_sfc/SX"
    sygro: str = "output_sfc/SY"
    szgro: str = "output_sfc/SZ"
    sxgro2: str = "output_vlm/SX"
    sygro2: str = "output_vlm/SY"
    szgro2: str = "output_vlm/SZ"
    sgtgro: str = "output_sgt/awp-strain"
    sgsn: str = "output_dyn/SGSN"

    def write(self, path: str):
        names = ["NBGX", "NEDX", "NSKPX", "NBGY", "NEDY", "NSKPY", "NBGZ", "NEDZ", "NSKPZ"]
        L = []
        L += ["%9d igreen" % self.igreen, "%9s TMAX" % self.tmax, "",
              "%9s DH" % self.dh, "%9s DT" % self.dt, "", "%9d NPC" % self.npc, "",
              "%9d ND" % self.nd, "%9s ARBC" % self.arbc, "%9s PHT" % self.pht, "",
              "%9d NSRC" % self.nsrc, "%9d NST" % self.nst, "",
              "%9d NX" % self.nx, "%9d NY" % self.ny, "%9d NZ" % self.nz, "",
              "%9d NPX" % self.npx, "%9d NPY" % self.npy, "%9d NPZ" % self.npz, ""]
        L += ["%9d IFAULT" % self.ifault, "%9d CHECKPOINT" % self.checkpoint, "%9d ISFCVLM" % self.isfcvlm,
              "%9d IMD5" % self.imd5, "%9d IVELOCITY" % self.ivelocity, "%9d MEDIARESTART" % self.mediarestart,
              "%9d NVAR" % self.nvar, "%9d IOST" % self.iost, "%9d PARTDEG" % self.partdeg,
              "%9d IO_OPT" % self.io_opt, "%9d PERF_MEAS" % self.perf_meas, "%9d IDYNA" % self.idyna,
              "%9d SOCALQ" % self.socalq, "", "%9d NVE" % self.nve, "",
              "%9s MU_S" % self.mu_s, "%9s MU_D" % self.mu_d, "",
              "%9s FL" % self.fl, "%9s FH" % self.fh, "%9s FP" % self.fp, "",
              "%9d READ_STEP" % self.read_step, "%9d WRITE_STEP" % self.write_step,
              "%9d WRITE_STEP2" % self.write_step2, ""]
        L += ["%9d %s" % (v, n) for v, n in zip(self.rec, names)]
        L += ["", "%9d NTISKP" % self.ntiskp, ""]
        L += ["%9d %s2" % (v, n) for v, n in zip(self.rec2, names)]
        L += ["", "%9d NTISKP2" % self.ntiskp2, "%9d NTISKP_SGT" % self.ntiskp_sgt, ""]
        L += ["'%s' CHKP" % self.chkp, "'%s' CHKJ" % self.chkj, "",
              "'%s' INSRC" % self.insrc, "'%s' INVEL" % self.invel, "", "'%s' INSGT" % self.insgt, "",
              "'%s' SXRGO" % self.sxgro, "'%s' SYRGO" % self.sygro, "'%s' SZRGO" % self.szgro, "",
              "'%s' SXRGO2" % self.sxgro2, "'%s' SYRGO2" % self.sygro2, "'%s' SZRGO2" % self.szgro2, "",
              "'%s' SGTGRO" % self.sgtgro, "", "'%s' SGSN" % self.sgsn]
        with open(path, "w") as f:
            f.write("\n".join(L) + "\n")

    @property
    def nt(self) -> int:
        x = np.float32(self.tmax) / np.float32(self.dt)
        return int(math.floor(float(x) + 0.5)) + 1


# ---------------------------------------------------------------------------
# benchmark configurations: the four CyberShake-style SGT workloads
# ---------------------------------------------------------------------------

@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    dh: float
    dt: float
    nst: int
    igreen: Tuple[int, ...]
    npts: int
    media_kind: str = "layered"
    src_xyz: Tuple[int, int, int] = (0, 0, 0)
    ntiskp_sgt: int = 10
    fl: float = 0.01
    fh: float = 25.0
    fp: float = 0.5
    socalq: int = 1
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def nt(self) -> int:
        return self.nst + 1

    def media(self) -> np.ndarray:
        if self.media_kind == "homogeneous":
            return homogeneous_media(self.nx, self.ny, self.nz)
        basin = self.extra.get("basin")
        return layered_media(self.nx, self.ny, self.nz, self.dh, self.seed, basin=basin)

    def points(self) -> np.ndarray:
        zmax = min(self.nz, max(1, int(round(10000.0 / self.dh)) + 1))
        return sgt_points(self.nx, self.ny, zmax, self.npts, seed=0)

    def stf(self, comp: int) -> np.ndarray:
        col = {1: 0, 2: 1, 3: 2}.get(self.igreen[comp], 0)
        return gaussian_derivative_stf(self.nst, self.dt, column=col)


def config(n: int) -> Workload:
    """Workload n (1..4) with its grid, steps and point count: 1 a 160x160x80
    homogeneous fx run, 2 a 400x400x200 layered fx+fy+fz run, 3 a 640x640x256
    layered fx+fy run, 4 a 1400x1000x400 basin fx+fy run."""
    if n == 1:
        return Workload("cfg1_homog_160x160x80_fx", 160, 160, 80, 200.0, 0.01, 1000, (1,), 1000,
                        media_kind="homogeneous", src_xyz=(80, 80, 11))
    if n == 2:
        return Workload("cfg2_layered_400x400x200_fxfyfz", 400, 400, 200, 100.0, 0.005, 4000, (1, 2, 3), 5000,
                        src_xyz=(200, 200, 21))
    if n == 3:
        return Workload("cfg3_layered_640x640x256_fxfy", 640, 640, 256, 100.0, 0.005, 3000, (1, 2), 5000,
                        src_xyz=(320, 320, 21))
    if n == 4:
        return Workload("cfg4_basin_1400x1000x400_fxfy", 1400, 1000, 400, 100.0, 0.005, 5000, (1, 2), 20000,
                        src_xyz=(700, 500, 21),
                        extra={"basin": {"cx": 70000.0, "cy": 50000.0, "rx": 30000.0, "ry": 20000.0,
                                         "depth": 4000.0}})
    raise ValueError(n)


# ---------------------------------------------------------------------------
# SGT header inputs (the files SgtHead's write_head reads)
# ---------------------------------------------------------------------------

def write_sgthead_inputs(d: str, nx: int, ny: int, nz: int, h_km: float, npts: int, seed: int = 0,
                         site=(None, None), mlon: float = -118.2, mlat: float = 34.05, mrot: float = -55.0,
                         edge_points: bool = True) -> dict:
    """Model box, RWG coordinate file, site location, grid file and AWP media
    file ([z][x][y][vp vs rho], y fastest, m/s and kg/m^3) for an nx x ny x nz
    RWG grid; returns the paths.  Points are distinct, seeded, and (with
    edge_points) include the special cases of the header writer: y = 0,
    x = nx-1, z = 0, z = 1 and z = nz-1."""
    os.makedirs(d, exist_ok=True)
    rng = np.random.default_rng(seed)
    paths = {k: os.path.join(d, k) for k in ("modelbox", "coordfile", "fdloc", "gridout", "media")}
    with open(paths["modelbox"], "w") as f:
        f.write("synthetic model box\nline 2\nline 3\nline 4\n")
        f.write("mlon= %.5f mlat= %.5f mrot= %.2f\n" % (mlon, mlat, mrot))
    xs, ys = site
    xs = nx // 2 if xs is None else xs
    ys = ny // 3 if ys is None else ys
    with open(paths["fdloc"], "w") as f:
        f.write("%d %d\n" % (xs, ys))
    with open(paths["gridout"], "w") as f:
        for name, n in (("x", nx), ("y", ny), ("z", nz)):
            f.write("%slen=%.6e\n%s=%d\n" % (name, n * h_km, "n" + name, n))
            for i in range(n):
                f.write("%d %12.5e %12.5e\n" % (i, i * h_km, h_km))
    pts = set()
    if edge_points:
        for p in ((0, 0, 0), (nx - 1, 3 % ny, 1), (2 % nx, 0, nz - 1), (nx - 1, ny - 1, nz - 1), (1, 1, 0)):
            pts.add(p)
    while len(pts) < npts:
        pts.add((int(rng.integers(0, nx)), int(rng.integers(0, ny)), int(rng.integers(0, nz))))
    pts = sorted(pts, key=lambda p: (p[1], p[0], p[2]))[:npts]
    with open(paths["coordfile"], "w") as f:
        f.write("# synthetic SGT coordinates\n# x y z indx lon lat dep\n%d\n" % len(pts))
        for x, y, z in pts:
            f.write("%d %d %d %d %.5f %.5f %.4f\n" % (x, y, z, x * 1000000000000 + y * 1000000 + z,
                                                     mlon + 0.01 * x, mlat + 0.01 * y, z * h_km))
    vs = (500.0 + 3500.0 * rng.random((nz, nx, ny))).astype(np.float32)
    vp = (1.73 * vs * (1.0 + 0.05 * rng.random((nz, nx, ny)))).astype(np.float32)
    rho = (310.0 * np.power(vp.astype(np.float64), 0.25)).astype(np.float32)
    np.stack([vp, vs, rho], axis=-1).astype(np.float32).tofile(paths["media"])
    return paths


# ---- reciprocity synthesis inputs -------------------------------------------

_GEO_RPERD = 0.017453292          # DirectSynth/src/jbsim/geoproj_subs.c:6
_GEO_ERAD = 6378.139


def _geo_matrices(alpha: float, lon: float, lat: float) -> np.ndarray:
    r = _GEO_RPERD
    ca, sa = math.cos(alpha * r), math.sin(alpha * r)
    ct, st = math.cos((90.0 - lat) * r), math.sin((90.0 - lat) * r)
    cp, sp = math.cos(lon * r), math.sin(lon * r)
    return np.array([ca * ct * cp + sa * sp, sa * ct * cp - ca * sp, st * cp,
                     ca * ct * sp - sa * cp, sa * ct * sp + ca * cp, st * sp,
                     -ca * st, -sa * st, ct])


def model_xy_to_lonlat(master, x_km, y_km):
    """Great-circle projection (geoproj 1) from model-frame km to degrees, the
    forward direction of geoproj_subs.c:10-77; float64, for placing points."""
    m = np.asarray(master).reshape(-1)[0]
    a = _geo_matrices(float(m["modelrot"]), float(m["modellon"]), float(m["modellat"]))
    g0 = 0.5 * (-2.0 * float(m["yshift"])) / _GEO_ERAD
    b0 = 0.5 * (-2.0 * float(m["xshift"])) / _GEO_ERAD
    x = np.asarray(x_km, np.float64)
    y = np.asarray(y_km, np.float64)
    cb, sb = np.cos(x / _GEO_ERAD - b0), np.sin(x / _GEO_ERAD - b0)
    cg, sg = np.cos(y / _GEO_ERAD - g0), np.sin(y / _GEO_ERAD - g0)
    arg = np.sqrt(1.0 + sb * sb * sg * sg)
    xp, yp = sg * cb * arg, sb * cg * arg
    zp = np.sqrt(1.0 - xp * xp - yp * yp)
    xg = xp * a[0] + yp * a[1] + zp * a[2]
    yg = xp * a[3] + yp * a[4] + zp * a[5]
    zg = xp * a[6] + yp * a[7] + zp * a[8]
    lat = 90.0 - np.arctan(np.sqrt(xg * xg + yg * yg) / zg) / _GEO_RPERD
    lon = np.where(xg != 0.0, np.arctan(yg / np.where(xg != 0.0, xg, 1.0)) / _GEO_RPERD, 0.0)
    lon = np.where(yg < 0.0, lon - 180.0, lon)
    return lon, lat


SYN_MASTER = np.dtype([("geoproj", "<i4"), ("modellon", "<f4"), ("modellat", "<f4"), ("modelrot", "<f4"),
                       ("xshift", "<f4"), ("yshift", "<f4"), ("globnp", "<i4"), ("localnp", "<i4"), ("nt", "<i4")])
SYN_INDEX = np.dtype([("indx", "<i8"), ("xsgt", "<i4"), ("ysgt", "<i4"), ("zsgt", "<i4"), ("h", "<f4")])
SYN_HEADER = np.dtype([("indx", "<i8"), ("geoproj", "<i4"), ("modellon", "<f4"), ("modellat", "<f4"),
                       ("modelrot", "<f4"), ("xshift", "<f4"), ("yshift", "<f4"), ("nt", "<i4"), ("xazim", "<f4"),
                       ("dt", "<f4"), ("tst", "<f4"), ("h", "<f4"), ("src_lat", "<f4"), ("src_lon", "<f4"),
                       ("src_dep", "<f4"), ("xsrc", "<i4"), ("ysrc", "<i4"), ("zsrc", "<i4"), ("sgt_lat", "<f4"),
                       ("sgt_lon", "<f4"), ("sgt_dep", "<f4"), ("xsgt", "<i4"), ("ysgt", "<i4"), ("zsgt", "<i4"),
                       ("cdist", "<f4"), ("lam", "<f4"), ("mu", "<f4"), ("rho", "<f4"), ("xmom", "<f4"),
                       ("ymom", "<f4"), ("zmom", "<f4")])
SYN_POINT = np.dtype([("lon", "<f4"), ("lat", "<f4"), ("dep", "<f4"), ("stk", "<f4"), ("dip", "<f4"),
                      ("area", "<f4"), ("tinit", "<f4"), ("dt", "<f4"), ("rake", "<f4"), ("slip1", "<f4"),
                      ("slip2", "<f4"), ("slip3", "<f4"), ("nt1", "<i4"), ("nt2", "<i4"), ("nt3", "<i4"),
                      ("stf1", "<i8"), ("stf2", "<i8"), ("stf3", "<i8")], align=True)


@dataclass
class SynthCase:
    master: np.ndarray
    index: np.ndarray
    headers: np.ndarray
    comps: List[np.ndarray]
    slon: float
    slat: float
    dtout: float
    ntout: int
    variations: List[Tuple[np.ndarray, np.ndarray]]
    h_km: float


def synth_case(seed: int = 0, nx_f: int = 12, nz_f: int = 6, nt: int = 300, nv: int = 3, ntout: int = 0,
               ncomp: int = 2, h_km: float = 1.0, dt: float = 0.1, drop_frac: float = 0.15,
               mech2_frac: float = 0.1, mech3_frac: float = 0.05, zero_frac: float = 0.05, nstf=(8, 40),
               jitter: float = 0.3, mrot: float = -55.0) -> SynthCase:
    """One site and one rupture in the formats DirectSynth reads: an SGT set
    (x-component master, index sorted by indx, headers, [np][6][nt] data per
    component) around a vertical fault of nx_f x nz_f points, and nv rupture
    variations on that fault.  A fraction of the fault's grid points is left
    out of the SGT set so that those rupture points take the four-point
    bracketing path; some points slip along u2 / u3 too, some not at all."""
    rng = np.random.default_rng(seed)
    nxm, nym = nx_f + 40, 60
    master = np.zeros(1, SYN_MASTER)
    master[0] = (1, -118.2, 34.05, mrot, -0.5 * nxm * h_km, -0.5 * nym * h_km, 0, 0, nt)
    xs, ys = 8, 10                                   # site (reciprocal source) grid location
    x0, yf = 20, 40                                  # fault trace start, fault y
    fault = [(x0 + i, yf, 1 + k) for i in range(nx_f) for k in range(nz_f)]
    drop = set(tuple(fault[i]) for i in rng.choice(len(fault), int(drop_frac * len(fault)), replace=False))
    pts = set()
    for x in range(x0 - 1, x0 + nx_f + 1):
        for y in (yf - 1, yf, yf + 1):
            for z in range(1, nz_f + 2):
                if (x, y, z) not in drop:
                    pts.add((x, y, z))
    pts = sorted(pts)
    npg = len(pts)
    master[0]["globnp"] = master[0]["localnp"] = npg
    index = np.zeros(npg, SYN_INDEX)
    p = np.array(pts, np.int64)
    index["indx"] = p[:, 0] * 1000000000000 + p[:, 1] * 1000000 + p[:, 2]
    index["xsgt"], index["ysgt"], index["zsgt"], index["h"] = p[:, 0], p[:, 1], p[:, 2], h_km
    hd = np.zeros(npg, SYN_HEADER)
    for f in ("geoproj", "modellon", "modellat", "modelrot", "xshift", "yshift", "nt"):
        hd[f] = master[0][f]
    hd["indx"], hd["xsgt"], hd["ysgt"], hd["zsgt"], hd["h"] = index["indx"], p[:, 0], p[:, 1], p[:, 2], h_km
    hd["xazim"], hd["dt"], hd["tst"] = 90.0 + mrot, dt, -4.0
    hd["xsrc"], hd["ysrc"], hd["zsrc"] = xs, ys, 1
    d = np.sqrt((p[:, 0] - xs) ** 2 + (p[:, 1] - ys) ** 2 + (p[:, 2] - 1) ** 2) * h_km
    hd["cdist"] = d
    vs = 3.0e5 * (1.0 + 0.1 * rng.random(npg))          # cm/s
    vp = 1.73 * vs
    rho = 2.4 + 0.3 * rng.random(npg)
    hd["rho"], hd["mu"], hd["lam"] = rho, rho * vs * vs, rho * (vp * vp - 2.0 * vs * vs)
    hd["xmom"] = 1.0e20
    t = (np.arange(nt) * dt).astype(np.float32)
    comps = []
    for q in range(ncomp):
        f0 = (0.2 + 0.8 * rng.random((npg, 6, 1))).astype(np.float32)
        td = ((d[:, None, None] / 3.0) + 2.0 * rng.random((npg, 6, 1))).astype(np.float32)
        amp = (1.0e-9 * (0.5 + rng.random((npg, 6, 1))) * np.where(rng.random((npg, 6, 1)) < 0.5, -1.0, 1.0)
               ).astype(np.float32)
        out = np.empty((npg, 6, nt), np.float32)
        for a in range(0, npg, 256):            # damped wavelets, 256 points at a time
            b = min(npg, a + 256)
            x = t[None, None, :] - td[a:b]
            out[a:b] = amp[a:b] * np.exp(-(x / 3.0) ** 2) * np.sin(np.float32(2.0 * np.pi) * f0[a:b] * x)
        comps.append(out)
    slon, slat = model_xy_to_lonlat(master, xs * h_km, ys * h_km)
    fx = np.array([f[0] for f in fault], np.float64) + jitter * (rng.random(len(fault)) - 0.5)
    fz = np.array([f[2] for f in fault], np.float64) + jitter * (rng.random(len(fault)) - 0.5)
    lon, lat = model_xy_to_lonlat(master, fx * h_km, np.full(len(fault), yf * h_km))
    variations = []
    nf = len(fault)
    for v in range(nv):
        sp = np.zeros(nf, SYN_POINT)
        sp["lon"], sp["lat"], sp["dep"] = lon, lat, (fz - 1.0) * h_km
        sp["stk"], sp["dip"] = 90.0 + mrot + 2.0 * (rng.random() - 0.5), 80.0 + 10.0 * rng.random()
        sp["area"] = (h_km * 1.0e5) ** 2
        sp["dt"] = dt
        sp["rake"] = 180.0 * (rng.random(nf) - 0.5) + 45.0 * v
        hyp = rng.integers(0, nf)
        sp["tinit"] = np.hypot(fx - fx[hyp], fz - fz[hyp]) * h_km / 2.8
        r = rng.random(nf)
        has = np.zeros((3, nf), bool)
        has[0] = r >= zero_frac
        has[1] = has[0] & (r < zero_frac + mech2_frac)
        has[2] = has[0] & (rng.random(nf) < mech3_frac)
        k = rng.integers(nstf[0], nstf[1] + 1, size=(nf, 3))
        slip = 20.0 + 200.0 * rng.random((nf, 3))
        pool, n = [], 0
        for i in range(nf):                      # samples of a point: u1, u2, u3 in order
            for c in range(3):
                if has[c, i]:
                    kk = int(k[i, c])
                    tri = np.minimum(np.arange(1, kk + 1), np.arange(kk, 0, -1)).astype(np.float64)
                    pool.append((slip[i, c] * tri / (tri.sum() * dt)).astype(np.float32))
                    sp[i]["slip%d" % (c + 1)], sp[i]["nt%d" % (c + 1)], sp[i]["stf%d" % (c + 1)] = slip[i, c], kk, n
                    n += kk
        variations.append((sp, np.concatenate(pool) if pool else np.zeros(0, np.float32)))
    return SynthCase(master, index, hd, comps, float(slon), float(slat), dt, ntout, variations, h_km)


def write_srf(path: str, pts: np.ndarray, pool: np.ndarray, binary: bool = False, plane: bool = True):
    """An SRF file (version 1.0) of the points, text or binary, in the layout
    DirectSynth/src/jbsim/srf_subs.c:521-690 reads."""
    if binary:
        with open(path, "wb") as f:
            f.write(b"1.0".ljust(32, b"\0"))
            if plane:
                f.write(b"PLANE".ljust(32, b"\0"))
                f.write(np.int32(1).tobytes())
                f.write(np.zeros(13, np.float32).tobytes())
            f.write(b"POINTS".ljust(32, b"\0"))
            f.write(np.int32(len(pts)).tobytes())
            for a in pts:
                f.write(np.array([a[k] for k in ("lon", "lat", "dep", "stk", "dip", "area", "tinit", "dt", "rake")],
                                 np.float32).tobytes())
                for c in (1, 2, 3):
                    f.write(np.float32(a["slip%d" % c]).tobytes() + np.int32(a["nt%d" % c]).tobytes())
                for c in (1, 2, 3):
                    n, o = int(a["nt%d" % c]), int(a["stf%d" % c])
                    f.write(pool[o:o + n].astype(np.float32).tobytes())
        return
    with open(path, "w") as f:
        f.write("1.0\n")
        if plane:
            f.write("PLANE 1\n%.5f %.5f %d %d %.2f %.2f\n%.1f %.1f %.2f %.2f %.2f\n" %
                    (-118.0, 34.0, 10, 5, 10.0, 5.0, 0.0, 90.0, 0.0, 0.0, 5.0))
        f.write("POINTS %d\n" % len(pts))
        for a in pts:
            f.write("%.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g\n" % tuple(
                float(a[k]) for k in ("lon", "lat", "dep", "stk", "dip", "area", "tinit", "dt")))
            f.write("%.9g %.9g %d %.9g %d %.9g %d\n" % (float(a["rake"]), float(a["slip1"]), int(a["nt1"]),
                                                      float(a["slip2"]), int(a["nt2"]), float(a["slip3"]),
                                                      int(a["nt3"])))
            for c in (1, 2, 3):
                n, o = int(a["nt%d" % c]), int(a["stf%d" % c])
                for j in range(0, n, 6):
                    f.write("  " + " ".join("%.9g" % float(x) for x in pool[o + j:o + min(n, j + 6)]) + "\n")
