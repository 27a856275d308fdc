"""Plasma / surface parameters (PAR) and model-selection flags (Flags), mirroring petch's
params.py key for key (petch/params.py:13-130) so existing configurations carry over unchanged.
Defaults are the ViennaPS SF6/O2 values the reference ships."""
from dataclasses import asdict, dataclass

import numpy as np

PAR = dict(
    ionFlux=12.0, Fflux=1800.0, Oflux=100.0,
    Emean=100.0, Esig=10.0,
    ion_ang_sigma=np.deg2rad(2.5),
    inflectAngle=1.55334303, minAngle=1.3962634, n_l=10.0,
    thetaRMin=np.deg2rad(70.0), thetaRMax=np.deg2rad(90.0),
    Eth_ie=15.0, Eth_sp=20.0, Eth_p=10.0,
    A_ie=7.0, A_sp=0.0337, A_p=3.0,
    s_F=0.20, s_O=0.30,
    rho=5.02,
    rate_scale=1.0,
    k_sigma=300.0,
    beta_sigma=0.04,
    B_sp=9.3,
    betaE=0.7,
    betaO=1.0,
    radiosity_solver='jacobi',
    knudsen_wall_loss_scale=2.9,
    knudsen_front_band_W=8.0,
    knudsen_passive_frac=0.5,
    knudsen_front_ar_pass=15.0,
    dda_n_dir=64,
    dda_n_reemit=12,
    ied_mode='mean',
    ied_dE=40.0,
    s_redep=0.5,
    k_redep=1.0,
    charge_alpha=0.0,
    eFlux=1.0,
    e_ang_sigma=0.5,
)


@dataclass
class Flags:
    """Model-selection toggles (petch/params.py:80-127); same names, values and defaults."""
    chemistry: str = "belen"
    yield_energy: str = "mean"
    yield_angular: str = "viennaps"
    ion_reflection: bool = False
    advection: str = "upwind1"
    sampling: str = "pseudo"
    transport_split: bool = False
    coverage_sticking: bool = False
    redeposition: bool = False
    neutral_transport: str = "mc"
    warm_start_coverage: bool = False
    surface_charging: object = False
    floor_charge_throttle: bool = False
    knudsen_front_loss: bool = False

    def to_dict(self):
        return asdict(self)


DEFAULT_FLAGS = Flags()
