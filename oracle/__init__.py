"""The oracle: a CPU FP64 restatement of CrowdPhot.jl's fitting hot path.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU legs (cpu_baseline and the reference arm) may import this package; the
product library (crowdphot.jl_b200/) never does.
"""
from .ffi import (orc_fit_simultaneous, orc_fit_star, orc_apply_J, orc_apply_JT, orc_lsqr_stamp, orc_lsqr_dense,
                  orc_lsmr_dense,
                  orc_ring_offsets, orc_morton2d, orc_bicubic, orc_psf_eval, orc_fill_stamps,
                  orc_model_radii_auto_gaussian, orc_exact_overlap, orc_aperture_weight, orc_unit_curve_of_growth,
                  orc_model_radii_auto, orc_fit_all_stars, orc_exp_disk_kernel, orc_spread_fwhm, orc_lm_irls_line,
                  orc_estimate_scale, orc_irls_weight, load)
