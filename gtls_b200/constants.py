"""Numerical constants of the TLS search.

Every value here is a data value the search depends on; each one equals the
reference's value so that grids, templates and defaults agree bit for bit.
Sources: ``src/gputls/constants.py`` (host constants, lines 33-171) and the
``#define`` block of the kernel source ``src/gputls/GPUFun.py:4-24`` (the
per-period duration-range constants, which differ from the host ones on
purpose in the reference and are kept apart here for that reason).
"""

VERSION = "0.1.0"
BANNER = "gtls_b200 " + VERSION + " (B200-native Transit Least Squares search)"

# astrophysical constants (constants.py:33-38)
G = 6.673e-11            # gravitational constant [m^3 / kg / s^2]
R_sun = 695508000        # [m]
R_earth = 6371000        # [m]
R_jup = 69911000         # [m]
M_sun = 1.989 * 10 ** 30  # [kg]
SECONDS_PER_DAY = 86400

# search defaults (constants.py:41-55)
TRANSIT_DEPTH_MIN = 10 * 10 ** -6
NUMERICAL_STABILITY_CUTOFF = 0.01 * 10 ** -6
R_STAR = 1.0
M_STAR = 1.0
OVERSAMPLING_FACTOR = 3
N_TRANSITS_MIN = 2
M_STAR_MIN = 0.1
M_STAR_MAX = 1.0
R_STAR_MIN = 0.13
R_STAR_MAX = 3.5
DURATION_GRID_STEP = 1.1

# reference transit template (constants.py:59-79)
DEFAULT_U = [0.4804, 0.1867]
DEFAULT_LIMB_DARK = "quadratic"
DEFAULT_ECC = 0
DEFAULT_W = 90
DEFAULT_PERIOD = 12.9
DEFAULT_RP = 0.03
DEFAULT_A = 23.1
DEFAULT_INC = 89.21
GRAZING_B = 0.99
BOX_PERIOD = 29
BOX_RP = 0.1
BOX_A = 26.9
BOX_B = 0
BOX_INC = 90
BOX_U = [0]
BOX_LIMB_DARK = "linear"
SIGNAL_DEPTH = 0.5
FRACTIONAL_TRANSIT_DURATION_MAX = 0.12
SUPERSAMPLE_SIZE = 10000
SDE_MEDIAN_KERNEL_SIZE = 30
T0_FIT_MARGIN = 0.125
MINIMUM_PERIOD_GRID_SIZE = 100

# per-period duration-range constants used on the device (GPUFun.py:8-24)
DEV_R_STAR_MIN = 0.05
DEV_R_STAR_MAX = 4.0
DEV_FRACTIONAL_TRANSIT_DURATION_MAX = 0.15
DEV_PI_GM_MAX = 416970
DEV_PI_GM_MIN = 20848
DEV_SCALE_FACTOR = 1000000000000000.0
# SKIP_POINT when T0_fit_margin == 0 (core.py:598-599): the bit pattern of
# +inf read as an int, i.e. "never skip".
SKIP_POINT_NEVER = 0x7F800000

# keyword arguments accepted by power() (constants.py:138-171)
VALID_PARAMETERS = [
    "R_star", "R_star_min", "R_star_max", "M_star", "M_star_min", "M_star_max",
    "period_min", "period_max", "periods", "n_transits_min", "GPUDeviceID",
    "GPUDeviceIDs", "legacy", "fast", "per", "rp", "a", "inc", "b", "ecc", "w",
    "u", "limb_dark", "duration_grid_step", "transit_depth_min",
    "oversampling_factor", "T0_fit_margin", "use_threads", "show_progress_bar",
    "transit_template", "verbose", "bar_location",
    # additions of this implementation (no counterpart in the reference)
    "precision", "batch_periods", "distributed", "useLocalPTXCUBIN", "refine",
]
