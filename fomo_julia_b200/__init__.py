"""fomo_julia_b200 -- B200 (sm_100a) engine for the time-stepping path of
Wuheng10086/Fomo_julia's Elastic2D module.

The compute lives in ``libfomo_b200.so`` (C ABI: ``include/fomo_b200.h``);
this package is the host-side mirror of the reference's API for that path.
"""
from .elastic2d import (  # noqa: F401
    AbstractBackend, B200Backend, B200_BACKEND, backend, to_device, synchronize, set_step_kernel,
    DeviceArray, Medium, HABCConfig, Wavefield, Source, Receivers, SimParams, sim_params,
    TimeStepInfo, ShotResult, ShotConfig, MultiShotConfig, multi_shot_config,
    get_fd_coefficients, ricker_wavelet, julia_mean, init_medium, init_medium_device, init_habc, setup_receivers,
    coord_to_index, create_source, reset, run_shot, run_shots, run_batch, save_gather, load_gather,
    pad_array, compute_staggered_params, taylor_coefficients,
)
from .serving import ShotServer, Ticket, percentile  # noqa: F401
from .snapshots import SnapshotRecorder, VideoConfig  # noqa: F401
from .geometry import (SurveyGeometry, MultiShotGeometry, create_geometry, save_geometry,  # noqa: F401
                       julia_str)

__version__ = "0.1.0"
