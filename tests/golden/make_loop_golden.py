"""Generates tests/golden/loop.npz: etch-depth histories of the oracle's loop (oracle/oracle.py
run_etch_3d, the FP64 restatement of petch's threed.py:1643-1795) on the benchmark
configurations, for the loop-level parity tests (tests/test_loop_configs_gpu.py).

    python tests/golden/make_loop_golden.py [case ...]

Cases (all SF6/O2 flags: Belen coverages, ViennaPS yields, faithful ions, coverage sticking,
warm-started coverage; FSM reinit; seed offset 0):

  c0_rs1      the hole of Process(Domain.hole(14, 0.25, 6, 2, 18), SF6O2(rate_scale=1.0),
              3.0).run(40): 56 x 56 x 96 grid, 30 000 rays per species, 40 steps (the front
              reaches the narrow-band speed limit and the domain floor)
  c0_rs025    the same hole at SF6O2's default rate_scale 0.025 (the front moves below the
              narrow-band limit, so the depth follows the fluxes)
  c1_mc       the 128 x 64 x 640 periodic trench (8 x 4 x 40 um, dx 0.0625, width 2, mask 1,
              sub_top 35), rate_scale 1.0, the first 30 steps of the 100-step 2.0 schedule,
              2^16 rays per species (MC neutrals)
  c1_mc_rs01  the same trench at rate_scale 0.1 (below the narrow-band limit)
  c1_rad      the same trench, neutral_transport='radiosity', rate_scale 1.0, 2^22 ions (the
              benchmark's count: the radiosity path does not smooth the ion yields, and at 2^16
              ions on ~5e4 faces the oracle's own runs with two seeds part by 8 cells)
  c1_rad_rs01 the same at rate_scale 0.1

Each case stores the oracle's centre depth after every step and the case's arguments (JSON).
Only the oracle runs here (no reference checkout is needed); the tests read the .npz.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (os.path.join(ROOT, "plasma-etching-code_b200"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import oracle.oracle as orc  # noqa: E402

SF6O2_FLAGS = dict(chemistry="belen", yield_angular="viennaps", coverage_sticking=True,
                   warm_start_coverage=True, sampling="sobol", ion_reflection=True)

C0 = dict(Lx=14.0, Ly=14.0, Lz=24.0, dx=0.25, trench_width=6.0, mask_th=2.0, sub_top=18.0,
          hole=True, t_end=3.0, n_steps=40)
C1 = dict(Lx=8.0, Ly=4.0, Lz=40.0, dx=0.0625, trench_width=2.0, mask_th=1.0, sub_top=35.0,
          hole=False, t_end=2.0 * 30 / 100, n_steps=30)

# par: overrides of PAR.  The config-0 cases carry SF6O2()'s parameter set (api.py:58-66: PAR
# with rate_scale and ied_mode "gauss"); the trench cases the benchmark's (PAR, periodic y).
CASES = {
    "c0_rs1": dict(geo=C0, par=dict(rate_scale=1.0, ied_mode="gauss", periodic_y=0),
                   rays=30000, transport="mc"),
    "c0_rs025": dict(geo=C0, par=dict(rate_scale=0.025, ied_mode="gauss", periodic_y=0),
                     rays=30000, transport="mc"),
    "c1_mc": dict(geo=C1, par=dict(rate_scale=1.0, periodic_y=1), rays=1 << 16, transport="mc"),
    "c1_mc_rs01": dict(geo=C1, par=dict(rate_scale=0.1, periodic_y=1), rays=1 << 16,
                       transport="mc"),
    "c1_rad": dict(geo=C1, par=dict(rate_scale=1.0, periodic_y=1), rays=1 << 22,
                   transport="radiosity"),
    "c1_rad_rs01": dict(geo=C1, par=dict(rate_scale=0.1, periodic_y=1), rays=1 << 22,
                        transport="radiosity"),
}


def run_case(case):
    from petch_b200 import params
    g = case['geo']
    par = dict(params.PAR, **case['par'])
    fl = params.Flags(neutral_transport=case['transport'], **SF6O2_FLAGS)
    t0 = time.time()
    _, hist, _ = orc.run_etch_3d(g['Lx'], g['Ly'], g['Lz'], g['dx'], g['trench_width'],
                                 g['mask_th'], g['sub_top'], g['t_end'], g['n_steps'], g['hole'],
                                 par, fl, case['rays'], case['rays'], record_depth_every=1)
    return np.array(hist, dtype=np.float64), time.time() - t0


def main(names):
    orc.build()
    path = os.path.join(HERE, "loop.npz")
    out = dict(np.load(path)) if os.path.exists(path) else {}
    for name in names:
        hist, sec = run_case(CASES[name])
        out[f"{name}_hist"] = hist
        out[f"{name}_case"] = np.array(json.dumps(CASES[name]))
        print(f"{name}: {sec:.1f} s, depth {hist[0, 1]:.3f} .. {hist[-1, 1]:.3f} um", flush=True)
    np.savez(path, **out)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
