"""The whole per-step loop through the drop-in API: the reference's own smoke tests
(tests/test_smoke.py in the reference, same configurations and assertions), and loop-level parity
with the oracle's etch loop: etch depth after N steps within one grid cell."""
import numpy as np
import pytest

import oracle.oracle as orc
import petch_b200 as petch
from petch_b200 import threed as t3

pytestmark = pytest.mark.gpu

SF6O2_FLAGS = dict(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                   warm_start_coverage=True, sampling="sobol", ion_reflection=True)


def test_reference_3d_loop():
    """Reference tests/test_smoke.py::test_3d_loop (trench, periodic y, 20 steps, 8000 rays)."""
    par = dict(petch.PAR)
    par['rate_scale'] = 0.1
    par['periodic_y'] = 1
    fl = petch.Flags(**SF6O2_FLAGS)
    geo = t3.run_etch_3d(Lx=3.0, Ly=0.9, Lz=6.5, dx=0.15, trench_width=0.9, mask_th=0.3,
                         sub_top=6.0, t_end=1.5, n_steps=20, par=par, flags=fl, n_ion=8000,
                         n_neu=8000, reinit_method="fsm", verbose=False)
    md, cd = t3.max_depth_3d(geo), t3.center_depth_3d(geo)
    assert np.isfinite(geo['phi']).all(), "level set blew up (non-finite phi)"
    assert md > 0.3, f"3D etch produced no depth (max_depth={md})"
    assert cd > 0.1, f"center did not etch (center_depth={cd}, max_depth={md})"


def test_reference_api_trench():
    """Reference tests/test_smoke.py::test_api_trench through Domain / SF6O2 / Process / Result."""
    dom = petch.Domain.trench(extent=3.0, dx=0.15, width=0.9, mask=0.3, depth=6.0)
    res = petch.Process(dom, petch.SF6O2(rate_scale=0.1), duration=1.5).run(steps=20)
    assert res.max_depth > 0.3, f"API etch shallow (max_depth={res.max_depth})"
    assert res.aspect_ratio > 0.3
    assert res.wall_time > 0.0
    v, f = res.mesh
    assert len(v) > 0 and len(f) > 0


def test_result_save_formats(tmp_path):
    dom = petch.Domain.hole(extent=4.0, dx=0.25, diameter=2.0, mask=1.0, depth=3.0, headroom=2.0)
    res = petch.Process(dom, petch.SF6O2(rate_scale=0.05), duration=0.5, n_ion=4000,
                        n_neu=4000).run(steps=3)
    v, f = res.mesh
    p = res.save(str(tmp_path / "s.vtk"))
    txt = open(p).read().splitlines()
    assert txt[0].startswith("# vtk") and f"POINTS {len(v)} float" in txt
    assert f"POLYGONS {len(f)} {4 * len(f)}" in txt
    p2 = res.save(str(tmp_path / "s.obj"))
    lines = open(p2).read().splitlines()
    assert sum(ln.startswith("v ") for ln in lines) == len(v)
    assert sum(ln.startswith("f ") for ln in lines) == len(f)


@pytest.mark.parametrize("hole", [True, False])
def test_loop_depth_matches_oracle_loop(hole):
    """Same configuration through the device engine and the oracle loop (independent random
    streams): centre depth within one grid cell at every recorded step."""
    dx = 0.25
    cfg = dict(Lx=5.0, Ly=5.0 if hole else 2.5, Lz=8.0, dx=dx, trench_width=2.0, mask_th=1.0,
               sub_top=6.0, t_end=1.2, n_steps=12, hole=hole)
    par = dict(petch.PAR, rate_scale=0.3, periodic_y=0 if hole else 1)
    fl = petch.Flags(**SF6O2_FLAGS)
    n = 60000
    geo = t3.run_etch_3d(**cfg, par=par, flags=fl, n_ion=n, n_neu=n, reinit_method="fsm",
                         verbose=False, record_depth_every=3)
    dev_hist = dict(geo['depth_history'])
    _, hist, _ = orc.run_etch_3d(cfg['Lx'], cfg['Ly'], cfg['Lz'], dx, cfg['trench_width'],
                                 cfg['mask_th'], cfg['sub_top'], cfg['t_end'], cfg['n_steps'],
                                 hole, par, fl, n, n, record_depth_every=3)
    orc_hist = dict(hist)
    assert set(dev_hist) == set(orc_hist)
    for s in sorted(orc_hist):
        assert abs(dev_hist[s] - orc_hist[s]) <= dx + 1e-9, (s, dev_hist[s], orc_hist[s])
    assert max(orc_hist.values()) > 2 * dx           # the feature actually etched
