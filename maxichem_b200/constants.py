"""Settings of the per-call chemistry solve: call limits, step control, guard, recovery and physical constants.

Every value here has the meaning and the value of the reference solver's setting of the same name
(imalsky/maxichem, ``maxichem/_constants.py:12-113``), because a drop-in replacement must refuse, step, guard and
recover exactly the cells the reference does. The CUDA kernels receive them through ``mx_settings`` (see
``include/maxichem_b200.h``); the CPU oracle receives the same struct, so one number is written once, here.
"""

# Call settings (maxichem/_constants.py:12-25).
T_MIN = 300.0  # K: colder cells are refused (counted "cold", not stepped)
T_MAX = 3000.0  # K: hotter cells are refused (counted "hot")
X_SUM_TOL = 1e-10  # |sum(x) - 1| above this is bad input, judged in the call kernel's own summation order
DRIFT = 1e-6  # default relative allowance on an element's share of the atoms over one call
REC_STEPS = 10  # the recovery's tries, in units of the call's max_steps
DEFAULT_RTOL = 1e-3
DEFAULT_MAX_STEPS = 4000
ATOL = 1e-25  # mole fraction

# Derivative settings (maxichem/_constants.py:28-29).
CAP = 100  # attempts a derivative call stores per cell before the adjoint checkpoints
DMAX = 16  # tangent directions per jvp call (MX_JVP_MAX_DIRECTIONS)
ARRHENIUS_COLUMNS = 9  # the rate table's differentiated columns: ln A, B, C of k0's two terms and of k_inf

# Reader limit (maxichem/_constants.py:36): largest |G/RT(low) - G/RT(high)| at NASA_SPLIT_T.
MAX_GIBBS_JUMP = 1.0e-5

# Method settings (maxichem/_constants.py:40-72).
H_MIN = 1e-12  # s: smallest first try of a call
CALL_END = 1.0 - 1e-14  # a call ends at this share of dt
STEP_SAFETY = 0.9
ERR_FLOOR = 1e-10
FAC_NONFINITE = 0.1
FACACC = 0.2
FACREJ = 0.2
FACMAX = 20.0
FAC_AFTER_REJECT = 0.5
SECMIN = 1e-4
SECANT_MIN_ORDER = 0.05
SECANT_MAX_ORDER = 3.0  # Rodas3's error order; the plain law takes its cube root
SECANT_TARGET = 0.5
PIVTAU = 0.1  # recovery: exchange rows only below this share of the column's largest entry
ELEMENT_PIVOT_MIN = 1e-10
REC_RETRIES = 3
REC_RETRY_SPLIT = 0.5
GMAX = 1e-3
NTAIL = 32  # rows of the dense trailing block, one per lane of the cell's warp

# Physical constants (maxichem/_constants.py:75-78).
KB = 1.380649e-16  # erg K^-1
P0 = 1.0e6  # dyn cm^-2: NASA-9 standard pressure
NASA_SPLIT_T = 1000.0  # K
K_COLL = 1e-9  # cm^3 s^-1: bimolecular-equivalent collision limit

# Rodas3 (Sandu et al. 1997), gamma = 1/2 (maxichem/kernels/common.cuh:5-7).
GAMMA = 0.5
RODAS_C21 = 4.0
RODAS_C43 = 8.0 / 3.0

# Troe factor coefficients (Venot et al. 2012, eq. C.2-C.5; maxichem/kernels/common.cuh:28-32).
TROE_C0 = 0.4
TROE_C1 = 0.67
TROE_N0 = 0.75
TROE_N1 = 1.27
TROE_D = 0.14

# Reaction kinds as VULCAN numbers them (maxichem/_constants.py:93-98).
KIND_TWO_BODY = 2
KIND_FALLOFF = 3
KIND_LOW_PRESSURE = 5
KIND_SPECIAL = 6
FALLOFF_KINDS = (KIND_FALLOFF, KIND_SPECIAL)
THREE_BODY_KINDS = (KIND_FALLOFF, KIND_LOW_PRESSURE, KIND_SPECIAL)

# Counts (maxichem/_constants.py:100-113): the device count array is queue, the ten COUNTS, recovery_queue.
COUNTS = (
    "bad_input",
    "cold",
    "hot",
    "nonfinite",
    "unfinished",
    "drift",
    "recomputed",
    "recovered",
    "still_failed",
    "nonfinite_h",
)
COUNT_SLOTS = ("queue", *COUNTS, "recovery_queue")

# Rate-law flag bits of a reaction (maxichem/_constants.py:117-129).
FL_FALLOFF = 1
FL_SECOND_K0 = 1 << 1
FL_THREE_BODY = 1 << 2
FL_TROE = 1 << 6
FL_EFF = 1 << 7
FL_VM11 = 1 << 9
FL_DMU_SHIFT = 3
FL_FORWARD_SHIFT = 10
FL_REVERSE_SHIFT = 12

# Status codes written by the screening (maxichem/kernels/common.cuh:260-262) and guard bits (guard.cuh:4-6).
REFUSED_COLD = 1
REFUSED_BAD_INPUT = 2
REFUSED_HOT = 3
GUARD_NONFINITE = 4
GUARD_UNFINISHED = 8
GUARD_DRIFT = 16

MAX_SPECIES = 254  # species indices are bytes, one value kept for the padding species
