"""Parity on the bench's own workload: 400x400x200, h = 100 m, dt = 5 ms,
fx+fy+fz stepped together by the default stepper (the staged sweeps, the
stress sweep with the three components side by side), 5000 SGT points, the
layered + 5 % perturbed medium; and on the 640x640x256 fx+fy workload the
same way (two components side by side, 5000 points).  With AWP_FULL_SIZE=1
also the 1400x1000x400 basin workload, fx+fy, 20000 points, whose FP32
state (78 GB) puts the default stress sweep on one component per work item;
it takes about 50 GB of host memory for the oracle and ten minutes, so it is
left out of the regular suite.

The solve starts from a state filled with bounded noise (every wavefield and
memory-variable cell of the interior; ghosts zero, as a solve keeps them), so
that every cell of every component is active from the first step on, and runs
60 steps with an SGT sample every 10.  Every field of every component, the
CHKJ series and the SGT file image must equal the FP32 oracle's bit for bit;
with the memory variables in block floating point ("bfp"), the FP32 oracle's
emulation of that storage.
"""
import os

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt
import oracle

pytestmark = pytest.mark.gpu

NT = 60
# magnitudes of the noise per state field: velocities, stresses, memory variables
SCALE = [1e-2] * 3 + [1e6] * 6 + [1e3] * 6


def noise(w, q, f):
    a = np.zeros((w.nz + 4, w.ny + 4, w.nx + 4), np.float32)
    rng = np.random.default_rng(1000 * (q + 1) + f)
    a[2:-2, 2:-2, 2:-2] = (rng.uniform(-1.0, 1.0, (w.nz, w.ny, w.nx)) * SCALE[f]).astype(np.float32)
    return a


SHAPES = {2: (400, 400, 200, 5000, (1, 2, 3)), 3: (640, 640, 256, 5000, (1, 2)),
          4: (1400, 1000, 400, 20000, (1, 2))}
full_size = pytest.mark.skipif(os.environ.get("AWP_FULL_SIZE") != "1", reason="AWP_FULL_SIZE=1 runs it")


@pytest.mark.parametrize("config,precision,rstore", [(2, "f32", "f32"), (2, "bfp", "bfp33"), (3, "f32", "f32"),
                                                     pytest.param(4, "f32", "f32", marks=full_size)])
def test_workload_bit_exact_from_a_noise_state(config, precision, rstore):
    w = ai.config(config)
    media = w.media()
    pts = w.points()
    assert (w.nx, w.ny, w.nz, len(pts), w.igreen) == SHAPES[config]
    nc = len(w.igreen)
    kw = dict(nd=20, arbc=0.92, fl=w.fl, fh=w.fh, fp=w.fp, socalq=w.socalq, ntiskp_sgt=10, write_step=6)
    stfs = [w.stf(q)[:NT] for q in range(nc)]
    p = awpsgt.make_params(w.nx, w.ny, w.nz, w.dh, w.dt, NT, igreen=w.igreen, nst=NT, precision=precision, **kw)
    with awpsgt.Solver(p) as s:
        tune = s.tuning()
        # components side by side in the stress sweep up to 32 GiB of state, one per item above
        assert bool(tune.staged_batch & 1) == (config != 4)
        s.load_media(media)
        for q in range(nc):
            s.set_source(q, [w.src_xyz], stfs[q])
        s.set_points(pts)
        start_r = []
        for q in range(nc):
            for f in range(15):
                s.set_field(awpsgt.FIELDS[f], noise(w, q, f), q)
            # the memory variables as stored (block floating point rounds them)
            start_r.append([s.field(awpsgt.FIELDS[f], q) for f in range(9, 15)] if precision != "f32" else None)
        s.run(NT)
        for q in range(nc):
            o = oracle.Oracle(nx=w.nx, ny=w.ny, nz=w.nz, dh=w.dh, dt=w.dt, nt=NT, nst=NT, igreen=w.igreen[q],
                              rstore=rstore, **kw)
            o.load_media(media)
            o.set_source([w.src_xyz], stfs[q])
            o.set_points(pts)
            for f in range(15):
                o.set_field(oracle.FIELDS[f], noise(w, q, f) if f < 9 or start_r[q] is None else start_r[q][f - 9])
            start_r[q] = None
            o.run(NT)
            bad = []
            for f in oracle.FIELDS[:15]:
                a, b = s.field(f, q), o.field(f)
                if not np.array_equal(a.view(np.uint32), b.view(np.uint32)):
                    bad.append((q, f, np.argwhere(a.view(np.uint32) != b.view(np.uint32))[0].tolist()))
            assert not bad, bad
            sg = s.sgt(q)
            assert sg.size == len(pts) * 6 * 6 and np.abs(sg).max() > 0
            assert np.array_equal(sg.view(np.uint32), o.sgt().view(np.uint32))
            assert np.array_equal(s.chkj(q).view(np.uint32), o.chkj().view(np.uint32))
            o.close()
