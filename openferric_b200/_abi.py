"""ctypes mirror of include/of_gpu.h (declarations only; nothing is loaded here).

Field order and widths must match the header exactly; tests/test_abi.py checks
the sizes against the compiled library's own view of them.
"""
import ctypes as C

OF_OK = 0
OF_ERR_INVALID_INPUT = 1
OF_ERR_NUMERICAL = 2
OF_ERR_CUDA = 3
OF_ERR_TIMEOUT = 4
OF_ERR_UNSUPPORTED = 5
OF_ERR_ALLOC = 6
OF_ERR_CONVERGENCE = 7

OF_CALL, OF_PUT = 0, 1
OF_MODEL_GBM, OF_MODEL_HESTON_EULER, OF_MODEL_HESTON_QE = 0, 1, 2
OF_PAYOFF_VANILLA, OF_PAYOFF_BARRIER, OF_PAYOFF_ASIAN = 0, 1, 2
OF_BARRIER_UP, OF_BARRIER_DOWN = 0, 1
OF_BARRIER_IN, OF_BARRIER_OUT = 0, 1
OF_AVG_ARITHMETIC, OF_AVG_GEOMETRIC = 0, 1
OF_STRIKE_FIXED, OF_STRIKE_FLOATING = 0, 1
OF_CV_NONE, OF_CV_VANILLA_TERMINAL, OF_CV_GEOMETRIC_ASIAN, OF_CV_TERMINAL_SPOT = 0, 1, 2, 3
OF_PREC_FP64_REFERENCE, OF_PREC_FP32_PHILOX = 0, 1


OF_DIV_CASH, OF_DIV_PROPORTIONAL = 0, 1


class OfDividendEvent(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("kind", C.c_int32),
        ("reserved0", C.c_int32),
        ("amount", C.c_double),
    ]


class OfModel(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved0", C.c_int32),
        ("s0", C.c_double),
        ("mu", C.c_double),
        ("sigma", C.c_double),
        ("maturity", C.c_double),
        ("steps", C.c_int64),
        ("kappa", C.c_double),
        ("theta", C.c_double),
        ("xi", C.c_double),
        ("rho", C.c_double),
        ("v0", C.c_double),
        ("dividends", C.POINTER(OfDividendEvent)),
        ("n_dividends", C.c_int64),
    ]


class OfPayoff(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("option_type", C.c_int32),
        ("strike", C.c_double),
        ("barrier_direction", C.c_int32),
        ("barrier_style", C.c_int32),
        ("barrier_level", C.c_double),
        ("rebate", C.c_double),
        ("averaging", C.c_int32),
        ("strike_type", C.c_int32),
        ("observation_times", C.POINTER(C.c_double)),
        ("n_observations", C.c_int64),
        ("expiry", C.c_double),
    ]


class OfMcConfig(C.Structure):
    _fields_ = [
        ("num_paths", C.c_int64),
        ("seed", C.c_uint64),
        ("antithetic", C.c_int32),
        ("precision", C.c_int32),
        ("control_variate", C.c_int32),
        ("tile_ilp", C.c_int32),
        ("cv_expected", C.c_double),
        ("discount_factor", C.c_double),
        ("injected_normals", C.POINTER(C.c_double)),
        ("n_injected", C.c_int64),
        ("rng_kind", C.c_int32),
        ("reserved0", C.c_int32),
    ]


OF_RNG_XOSHIRO256PP, OF_RNG_PCG64 = 0, 1


class OfBookEntry(C.Structure):
    _fields_ = [
        ("model", OfModel),
        ("payoff", OfPayoff),
        ("num_paths", C.c_int64),
        ("antithetic", C.c_int32),
        ("control_variate", C.c_int32),
        ("cv_expected", C.c_double),
        ("discount_factor", C.c_double),
    ]


OF_BOOK_PRICE = 0
OF_BOOK_GREEKS = 1
OF_BOOK_PRICE_FP64 = 2
OF_BOOK_GREEKS_FP64 = 3


class OfBookConfig(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("block", C.c_int32),
        ("paths_per_thread", C.c_int32),
        ("use_graph", C.c_int32),
        ("mode", C.c_int32),
    ]


class OfBookGreeks(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("delta", "gamma", "vega", "theta", "rho",
                                           "delta_se", "gamma_se", "vega_se", "theta_se", "rho_se")]


class OfStderrTarget(C.Structure):
    _fields_ = [
        ("se_rel", C.c_double),
        ("pilot_paths", C.c_int64),
        ("max_rounds", C.c_int32),
        ("reserved0", C.c_int32),
        ("margin", C.c_double),
    ]


class OfStderrRound(C.Structure):
    _fields_ = [
        ("options", C.c_int64),
        ("paths", C.c_int64),
        ("path_steps", C.c_double),
        ("converged", C.c_int64),
        ("kernel_ms", C.c_double),
        ("wall_ms", C.c_double),
    ]


class OfTuneCandidate(C.Structure):
    _fields_ = [
        ("block", C.c_int32),
        ("paths_per_thread", C.c_int32),
        ("ms", C.c_double),
    ]


class OfGreeksParams(C.Structure):
    _fields_ = [
        ("option_type", C.c_int32),
        ("antithetic", C.c_int32),
        ("spot", C.c_double),
        ("strike", C.c_double),
        ("rate", C.c_double),
        ("dividend_yield", C.c_double),
        ("vol", C.c_double),
        ("expiry", C.c_double),
        ("num_paths", C.c_int64),
        ("num_steps", C.c_int64),
        ("seed", C.c_uint64),
        ("spot_bump_rel", C.c_double),
        ("mu", C.c_double),
        ("kappa", C.c_double),
        ("theta", C.c_double),
        ("xi", C.c_double),
        ("rho", C.c_double),
        ("v0", C.c_double),
    ]


class OfGreeksResult(C.Structure):
    _fields_ = [
        ("price", C.c_double),
        ("stderr_", C.c_double),
        ("delta", C.c_double),
        ("gamma", C.c_double),
        ("vega", C.c_double),
        ("theta", C.c_double),
        ("rho", C.c_double),
        ("lr_delta", C.c_double),
        ("lr_gamma", C.c_double),
        ("lr_vega", C.c_double),
        ("samples", C.c_int64),
        ("kernel_ms", C.c_double),
    ]


OF_EXERCISE_EUROPEAN, OF_EXERCISE_AMERICAN, OF_EXERCISE_BERMUDAN = 0, 1, 2


class OfLsmContract(C.Structure):
    _fields_ = [
        ("option_type", C.c_int32),
        ("exercise", C.c_int32),
        ("spot", C.c_double),
        ("strike", C.c_double),
        ("rate", C.c_double),
        ("dividend_yield", C.c_double),
        ("vol", C.c_double),
        ("expiry", C.c_double),
        ("num_steps", C.c_int64),
        ("exercise_dates", C.POINTER(C.c_double)),
        ("n_exercise_dates", C.c_int64),
    ]


class OfLsmBarrierContract(C.Structure):
    _fields_ = [
        ("option_type", C.c_int32),
        ("barrier_direction", C.c_int32),
        ("barrier_style", C.c_int32),
        ("reserved0", C.c_int32),
        ("spot", C.c_double),
        ("strike", C.c_double),
        ("rate", C.c_double),
        ("dividend_yield", C.c_double),
        ("vol", C.c_double),
        ("expiry", C.c_double),
        ("barrier_level", C.c_double),
        ("rebate", C.c_double),
        ("num_steps", C.c_int64),
    ]


class OfLsmConfig(C.Structure):
    _fields_ = [
        ("num_paths", C.c_int64),
        ("seed", C.c_uint64),
        ("precision", C.c_int32),
        ("basis_degree", C.c_int32),
        ("want_delta", C.c_int32),
        ("batch_contracts", C.c_int32),
        ("injected_normals", C.POINTER(C.c_double)),
        ("n_injected", C.c_int64),
    ]


class OfLsmResult(C.Structure):
    _fields_ = [
        ("price", C.c_double),
        ("stderr_", C.c_double),
        ("delta", C.c_double),
        ("regressions", C.c_int64),
        ("kernel_ms", C.c_double),
    ]


OF_ADJ_NAMES = ("spot", "rate", "v0", "kappa", "theta", "xi", "rho")


class OfHestonAdjointParams(C.Structure):
    _fields_ = [
        ("spot", C.c_double),
        ("strike", C.c_double),
        ("rate", C.c_double),
        ("dividend_yield", C.c_double),
        ("expiry", C.c_double),
        ("kappa", C.c_double),
        ("theta", C.c_double),
        ("xi", C.c_double),
        ("rho", C.c_double),
        ("v0", C.c_double),
        ("num_paths", C.c_int64),
        ("num_steps", C.c_int64),
        ("seed", C.c_uint64),
        ("option_type", C.c_int32),
        ("payoff", C.c_int32),
        ("scheme", C.c_int32),
        ("checkpoint_every", C.c_int32),
        ("forward_only", C.c_int32),
        ("reserved0", C.c_int32),
        ("qe_switch_band", C.c_double),
    ]


class OfAdjointResult(C.Structure):
    _fields_ = [
        ("price", C.c_double),
        ("stderr_", C.c_double),
        ("greeks", C.c_double * 7),
        ("greeks_stderr", C.c_double * 7),
        ("samples", C.c_int64),
        ("kernel_ms", C.c_double),
    ]


class OfMcResult(C.Structure):
    _fields_ = [
        ("price", C.c_double),
        ("stderr_", C.c_double),
        ("samples", C.c_int64),
        ("sum_x", C.c_double),
        ("sum_x2", C.c_double),
        ("sum_y", C.c_double),
        ("sum_xy", C.c_double),
        ("sum_y2", C.c_double),
        ("kernel_ms", C.c_double),
    ]


class OfDevicePeaks(C.Structure):
    _fields_ = [
        ("sfu_ops_per_s", C.c_double),
        ("fp32_flops_per_s", C.c_double),
        ("probe_ms", C.c_double),
        ("fp64_flops_per_s", C.c_double),
    ]


OF_LSM_GBM, OF_LSM_LOCAL_VOL, OF_LSM_HESTON_EULER = 0, 1, 2


class OfBermudanContract(C.Structure):
    _fields_ = [
        ("option_type", C.c_int32),
        ("dynamics", C.c_int32),
        ("spot", C.c_double),
        ("rate", C.c_double),
        ("dividend_yield", C.c_double),
        ("vol", C.c_double),
        ("expiry", C.c_double),
        ("num_steps", C.c_int64),
        ("schedule_times", C.POINTER(C.c_double)),
        ("schedule_strikes", C.POINTER(C.c_double)),
        ("n_schedule", C.c_int64),
        ("lv_strikes", C.POINTER(C.c_double)),
        ("lv_n_strikes", C.c_int64),
        ("lv_expiries", C.POINTER(C.c_double)),
        ("lv_n_expiries", C.c_int64),
        ("lv_vols", C.POINTER(C.c_double)),
        ("kappa", C.c_double),
        ("theta", C.c_double),
        ("xi", C.c_double),
        ("rho", C.c_double),
        ("v0", C.c_double),
    ]


class OfBoundaryPoint(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("strike", C.c_double),
        ("boundary_spot", C.c_double),
        ("has_boundary", C.c_int32),
        ("reserved0", C.c_int32),
        ("itm_paths", C.c_int64),
        ("exercised_paths", C.c_int64),
    ]


class OfQmcParams(C.Structure):
    _fields_ = [
        ("option_type", C.c_int32),
        ("precision", C.c_int32),
        ("spot", C.c_double),
        ("strike", C.c_double),
        ("rate", C.c_double),
        ("dividend_yield", C.c_double),
        ("vol", C.c_double),
        ("expiry", C.c_double),
        ("num_paths", C.c_int64),
        ("num_steps", C.c_int64),
        ("seed", C.c_uint64),
    ]
