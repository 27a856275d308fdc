"""Host-side pieces of the batched forward (CPU only)."""
import numpy as np

from petch_b200.batch import hole_batch_specs


def test_hole_batch_specs_follow_the_ragged_distribution():
    specs = hole_batch_specs(64, seed=0)
    d = np.array([s['trench_width'] for s in specs])
    m = np.array([s['mask_th'] for s in specs])
    E = np.array([s['par']['Emean'] for s in specs])
    assert d.min() >= 2.0 and d.max() <= 8.0 and m.min() >= 1.0 and m.max() <= 3.0
    assert E.min() >= 50.0 and E.max() <= 500.0
    nx = [round(s['Lx'] / s['dx']) for s in specs]
    assert min(nx) >= 40 and max(nx) <= 64
    assert all(round(s['Lz'] / s['dx']) == 96 for s in specs)
