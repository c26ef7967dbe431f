"""Hot-path options and their defaults.

The option names, types and defaults are those of the reference's argparse
sections (src/tomocupy/config.py:104-600) for every flag the reconstruction
path reads; file-I/O, CLI and logging options are out of scope.  Unknown keys
passed to :func:`make_args` raise, unlike the reference's silent
``parse_known_args``.
"""
from __future__ import annotations

from argparse import Namespace

DEFAULTS = {
    # reconstruction (config.py:310-450)
    "reconstruction_type": "full",          # 'full' | 'try' | 'try_lamino'
    "reconstruction_algorithm": "fourierrec",  # 'fourierrec' | 'lprec' | 'linerec'
    "fbp_filter": "parzen",
    "dtype": "float32",                     # 'float32' | 'float16' | 'mixed' (tensor-core filter)
    "out_dtype": "float32",                 # 'float32' | 'float16' output slices (fourierrec)
    "mixed_filter": "fft",                  # dtype 'mixed': 'fft' (fused fp32) | 'tensor' (tcgen05)
    "rotation_axis": -1.0,
    "center_search_width": 50.0,
    "center_search_step": 0.5,
    "nsino": "0.5",
    "nsino_per_chunk": 8,
    "nproj_per_chunk": 8,
    "start_row": 0,
    "end_row": -1,
    "start_column": 0,
    "end_column": -1,
    "start_proj": 0,
    "end_proj": -1,
    "binning": 0,
    "blocked_views": "none",
    "file_type": "standard",
    # pre-processing
    "minus_log": "True",
    "bright_ratio": 1.0,
    "flat_linear": "False",
    "dezinger": 0,
    "dezinger_threshold": 5000,
    "remove_stripe_method": "none",         # 'none' | 'fw' | 'ti' | 'vo-all'
    "fw_sigma": 1.0,
    "fw_filter": "sym16",
    "fw_level": 7,
    "fw_pad": True,
    "ti_beta": 0.022,
    "ti_mask": 1.0,
    "vo_all_snr": 3.0,
    "vo_all_la_size": 61,
    "vo_all_sm_size": 21,
    "vo_all_dim": 1,
    "retrieve_phase_method": "none",        # 'none' | 'paganin' | 'Gpaganin' | 'farago'
    "energy": 20.0,                         # keV
    "propagation_distance": 0.0,            # mm
    "pixel_size": 0.0,                      # microns
    "retrieve_phase_alpha": 0.0,
    "retrieve_phase_delta_beta": 1500.0,
    "retrieve_phase_W": 2e-4,               # microns
    "retrieve_phase_pad": 1,
    "rotate_proj_angle": 0.0,
    "rotate_proj_order": 1,
    "beam_hardening_method": "none",
    # laminography
    "lamino_angle": 0.0,
    "lamino_start_row": 0,
    "lamino_end_row": -1,
    "lamino_search_width": 5.0,
    "lamino_search_step": 0.25,
    # steps API
    "pre_processing": "True",
    "max_write_threads": 4,
    "max_read_threads": 1,
}


def make_args(**overrides) -> Namespace:
    """A fresh args namespace with the reference defaults and the given overrides."""
    unknown = set(overrides) - set(DEFAULTS)
    if unknown:
        raise KeyError(f"unknown option(s): {sorted(unknown)}")
    d = dict(DEFAULTS)
    d.update(overrides)
    return Namespace(**d)
