"""B200-native WaveQ3D wavefront propagation engine.

A drop-in for USML's ``usml::waveq3d::wave_queue`` path: the classes here
keep the reference names (``wave_queue``, ``ocean_model``, ``profile_munk``,
``boundary_flat``, ``seq_rayfan``, ``eigenray_collection`` ...) while all
propagation runs in hand-written sm_100a CUDA kernels inside
``libwq3d.so`` (C ABI: ``include/wq3d.h``).  There is no CPU fallback.
"""
from . import _abi
from .types import (seq_vector, seq_linear, seq_log, seq_data, seq_rayfan,
                    wposition, wposition1, compute_earth_radius, earth_radius,
                    set_earth_radius, to_degrees, to_radians)
from .ocean import (attenuation_thorp, attenuation_constant, profile_linear,
                    profile_munk, profile_catenary, profile_n2, reflect_loss_constant,
                    reflect_loss_rayleigh, reflect_loss_eckart, boundary_flat,
                    boundary_slope, ocean_model, data_grid, profile_grid, boundary_grid,
                    volume_flat, scattering_constant, scattering_lambert, scattering_chapman)
from .waveq3d import (wave_queue, eigenray_listener, reflection_listener,
                      eigenray_model, eigenray_list, run_batch)
from .eigenrays import eigenray_collection
from .wavegen import run_wavefront_generators, wavefront_generator
from .eigenverbs import eigenverb_model, eigenverb_listener, eigenverb_collection
from .biverbs import biverb_model, biverb_collection, biverb_generator

load_engine = _abi.load_engine
EngineError = _abi.EngineError
LIB_PATH = _abi.LIB_PATH

__all__ = [
    "seq_vector", "seq_linear", "seq_log", "seq_data", "seq_rayfan", "wposition",
    "wposition1", "compute_earth_radius", "earth_radius", "set_earth_radius",
    "to_degrees", "to_radians", "attenuation_thorp", "attenuation_constant",
    "profile_linear", "profile_munk", "profile_catenary", "profile_n2",
    "reflect_loss_constant", "reflect_loss_rayleigh", "reflect_loss_eckart",
    "boundary_flat", "boundary_slope", "ocean_model", "data_grid", "profile_grid",
    "boundary_grid", "volume_flat", "scattering_constant", "scattering_lambert",
    "scattering_chapman", "wave_queue", "run_batch",
    "eigenray_listener", "reflection_listener", "eigenray_model", "eigenray_list",
    "wavefront_generator", "run_wavefront_generators",
    "eigenray_collection", "eigenverb_model", "eigenverb_listener", "eigenverb_collection",
    "biverb_model", "biverb_collection", "biverb_generator",
    "load_engine", "EngineError", "LIB_PATH",
]
