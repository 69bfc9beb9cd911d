"""ctypes wrapper of the CPU oracle (liboforacle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product package never
imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from openferric_b200._abi import OfMcConfig, OfMcResult, OfModel, OfPayoff

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboforacle.so")
_lib = None

D = C.c_double
I64 = C.c_int64
PD = C.POINTER(C.c_double)


def build():
    """Compiles the oracle with its Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_acklam_inv_cdf.restype = D
        L.orc_acklam_inv_cdf.argtypes = [D]
        L.orc_hart_norm_cdf.restype = D
        L.orc_hart_norm_cdf.argtypes = [D]
        L.orc_uniform_open01.restype = D
        L.orc_uniform_open01.argtypes = [D]
        L.orc_stream_seed.restype = C.c_uint64
        L.orc_stream_seed.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_xoshiro_seed.argtypes = [C.c_void_p, C.c_uint64]
        L.orc_xoshiro_next_u64.restype = C.c_uint64
        L.orc_xoshiro_next_u64.argtypes = [C.c_void_p]
        L.orc_xoshiro_next_f64.restype = D
        L.orc_xoshiro_next_f64.argtypes = [C.c_void_p]
        L.orc_pcg64_seed.argtypes = [C.c_void_p, C.c_uint64]
        L.orc_pcg64_next_u64.restype = C.c_uint64
        L.orc_pcg64_next_u64.argtypes = [C.c_void_p]
        L.orc_fill_run_normals.argtypes = [C.c_uint64, I64, I64, C.c_int, PD]
        L.orc_fill_sequential_normals.argtypes = [C.c_uint64, I64, PD]
        L.orc_bs_price.restype = D
        L.orc_bs_price.argtypes = [C.c_int, D, D, D, D, D, D]
        L.orc_bs_greeks.argtypes = [C.c_int, D, D, D, D, D, D] + [PD] * 5
        L.orc_geometric_asian_discrete_fixed.restype = D
        L.orc_geometric_asian_discrete_fixed.argtypes = [C.c_int, D, D, D, D, D, PD, I64]
        L.orc_heston_call.restype = D
        L.orc_heston_call.argtypes = [D] * 10
        L.orc_heston_put.restype = D
        L.orc_heston_put.argtypes = [D] * 10
        L.orc_crr_american.restype = D
        L.orc_crr_american.argtypes = [C.c_int, D, D, D, D, D, D, I64]
        L.orc_mc_run.restype = C.c_int
        L.orc_mc_run.argtypes = [C.POINTER(OfModel), C.POINTER(OfPayoff), C.POINTER(OfMcConfig), C.c_int,
                                 C.POINTER(OfMcResult)]
        L.orc_mc_strip.restype = C.c_int
        L.orc_mc_strip.argtypes = [C.POINTER(OfModel), C.c_int, PD, I64, C.POINTER(OfMcConfig), C.c_int,
                                   C.POINTER(OfMcResult)]
        L.orc_generate_path.argtypes = [C.POINTER(OfModel), PD, PD, PD]
        L.orc_payoff_from_path.restype = D
        L.orc_payoff_from_path.argtypes = [C.POINTER(OfPayoff), PD, I64]
        L.orc_gbm_pathwise_aad.restype = C.c_int
        L.orc_gbm_pathwise_aad.argtypes = [C.c_int, D, D, D, D, D, D, I64, I64, C.c_uint64, C.c_int, PD]
        L.orc_heston_price_delta.restype = C.c_int
        L.orc_heston_price_delta.argtypes = [C.c_int] + [D] * 10 + [I64, I64, C.c_uint64, PD]
        L.orc_mc_greek_estimators.restype = C.c_int
        L.orc_mc_greek_estimators.argtypes = [C.c_int, D, D, D, D, D, D, I64, C.c_uint64, C.c_int, D, PD]
        L.orc_lsm_price.restype = C.c_int
        L.orc_lsm_price.argtypes = [C.c_int, D, D, C.c_int, PD, I64, D, D, D, D, I64, I64, C.c_uint64, C.c_int,
                                    PD, PD]
        L.orc_sobol_dimension.restype = None
        L.orc_sobol_dimension.argtypes = [C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.orc_sobol_points.restype = C.c_int
        L.orc_sobol_points.argtypes = [I64, C.c_uint64, I64, PD]
        L.orc_mc_european_qmc.restype = C.c_int
        L.orc_mc_european_qmc.argtypes = [C.c_int, D, D, D, D, D, D, I64, I64, C.c_uint64, PD]
        L.orc_sampled_vol.restype = D
        L.orc_sampled_vol.argtypes = [PD, I64, PD, I64, PD, D, D]
        L.orc_lsm_bermudan.restype = C.c_int
        L.orc_lsm_bermudan.argtypes = ([C.c_int, D, PD, PD, I64, C.c_int, D, D, D, D, PD, I64, PD, I64, PD] + [D] * 5 +
                                       [I64, I64, C.c_uint64, C.c_int, PD, PD, PD, C.POINTER(I64)])
        L.orc_wgsl_european.restype = C.c_int
        L.orc_wgsl_european.argtypes = [D, D, D, D, D, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, PD, PD]
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(PD) if a is not None else None


class Xoshiro:
    def __init__(self, seed):
        self._state = (C.c_uint64 * 4)()
        lib().orc_xoshiro_seed(C.byref(self._state), C.c_uint64(seed))

    def next_u64(self):
        return lib().orc_xoshiro_next_u64(C.byref(self._state))

    def next_f64(self):
        return lib().orc_xoshiro_next_f64(C.byref(self._state))

    def state(self):
        return list(self._state)


class Pcg64:
    """The C oracle's Pcg64 (two 128-bit words: state, increment)."""

    def __init__(self, seed):
        self._state = (C.c_uint64 * 4)()
        lib().orc_pcg64_seed(C.byref(self._state), C.c_uint64(seed))

    def next_u64(self):
        return lib().orc_pcg64_next_u64(C.byref(self._state))


def acklam(p):
    return lib().orc_acklam_inv_cdf(p)


def hart_cdf(x):
    return lib().orc_hart_norm_cdf(x)


def run_normals(seed, samples, steps, streams):
    out = np.empty(samples * steps * streams, dtype=np.float64)
    lib().orc_fill_run_normals(seed, samples, steps, streams, _ptr(out))
    return out


def sequential_normals(seed, count):
    out = np.empty(count, dtype=np.float64)
    lib().orc_fill_sequential_normals(seed, count, _ptr(out))
    return out


def bs_price(option_type, spot, strike, rate, q, vol, expiry):
    return lib().orc_bs_price(option_type, spot, strike, rate, q, vol, expiry)


def bs_greeks(option_type, spot, strike, rate, q, vol, expiry):
    o = [D() for _ in range(5)]
    lib().orc_bs_greeks(option_type, spot, strike, rate, q, vol, expiry, *[C.byref(x) for x in o])
    return dict(zip(["delta", "gamma", "vega", "theta", "rho"], [x.value for x in o]))


def geometric_asian(option_type, s0, k, r, q, sigma, obs):
    obs = np.ascontiguousarray(obs, dtype=np.float64)
    return lib().orc_geometric_asian_discrete_fixed(option_type, s0, k, r, q, sigma, _ptr(obs), len(obs))


def heston_call(s0, k, r, q, T, v0, kappa, theta, xi, rho):
    return lib().orc_heston_call(s0, k, r, q, T, v0, kappa, theta, xi, rho)


def heston_put(s0, k, r, q, T, v0, kappa, theta, xi, rho):
    return lib().orc_heston_put(s0, k, r, q, T, v0, kappa, theta, xi, rho)


def crr_american(option_type, s0, k, r, q, vol, T, steps):
    return lib().orc_crr_american(option_type, s0, k, r, q, vol, T, steps)


def mc_run(model, payoff, cfg, threads=1):
    out = OfMcResult()
    st = lib().orc_mc_run(C.byref(model), C.byref(payoff), C.byref(cfg), threads, C.byref(out))
    if st != 0:
        raise RuntimeError(f"orc_mc_run status {st}")
    return out


def mc_strip(model, option_type, strikes, cfg, threads=1):
    strikes = np.ascontiguousarray(strikes, dtype=np.float64)
    out = (OfMcResult * len(strikes))()
    st = lib().orc_mc_strip(C.byref(model), option_type, _ptr(strikes), len(strikes), C.byref(cfg), threads, out)
    if st != 0:
        raise RuntimeError(f"orc_mc_strip status {st}")
    return list(out)


def generate_path(model, z1, z2=None):
    z1 = np.ascontiguousarray(z1, dtype=np.float64)
    z2 = np.ascontiguousarray(z2 if z2 is not None else np.zeros_like(z1), dtype=np.float64)
    path = np.empty(model.steps + 1, dtype=np.float64)
    lib().orc_generate_path(C.byref(model), _ptr(z1), _ptr(z2), _ptr(path))
    return path


def gbm_pathwise_aad(option_type, strike, spot, rate, q, vol, expiry, num_paths, num_steps, seed, antithetic):
    out = np.zeros(6)
    st = lib().orc_gbm_pathwise_aad(option_type, strike, spot, rate, q, vol, expiry, num_paths, num_steps, seed,
                                    int(antithetic), _ptr(out))
    if st != 0:
        raise RuntimeError(f"orc_gbm_pathwise_aad status {st}")
    return dict(zip(["price", "stderr", "delta", "vega", "theta", "rho"], out.tolist()))


def heston_price_delta(option_type, strike, maturity, spot, rate, mu, kappa, theta, xi, rho, v0, num_paths,
                       num_steps, seed):
    out = np.zeros(2)
    st = lib().orc_heston_price_delta(option_type, strike, maturity, spot, rate, mu, kappa, theta, xi, rho, v0,
                                      num_paths, num_steps, seed, _ptr(out))
    if st != 0:
        raise RuntimeError(f"orc_heston_price_delta status {st}")
    return float(out[0]), float(out[1])


def mc_greek_estimators(option_type, strike, spot, rate, q, vol, expiry, num_paths, seed, antithetic=True,
                        spot_bump_rel=1e-2):
    out = np.zeros(5)
    st = lib().orc_mc_greek_estimators(option_type, strike, spot, rate, q, vol, expiry, num_paths, seed,
                                       int(antithetic), spot_bump_rel, _ptr(out))
    if st != 0:
        raise RuntimeError(f"orc_mc_greek_estimators status {st}")
    return dict(zip(["pathwise_delta", "pathwise_gamma", "lr_delta", "lr_gamma", "lr_vega"], out.tolist()))


def lsm_barrier(option_type, strike, expiry, up, knock_in, level, rebate, spot, rate, q, vol, num_paths, num_steps,
                seed, normals=None):
    """LongstaffSchwartzEngine::price(BarrierOption) restated: (price, stderr)."""
    L = lib()
    f = L.orc_lsm_barrier
    f.restype = C.c_int
    f.argtypes = [C.c_int, D, D, C.c_int, C.c_int, D, D, D, D, D, D, I64, I64, C.c_uint64, PD, PD]
    out = np.zeros(2)
    z = None if normals is None else np.ascontiguousarray(normals, dtype=np.float64)
    st = f(option_type, strike, expiry, int(up), int(knock_in), level, rebate, spot, rate, q, vol, num_paths,
           num_steps, seed, _ptr(z) if z is not None else None, _ptr(out))
    if st != 0:
        raise RuntimeError(f"orc_lsm_barrier status {st}")
    return float(out[0]), float(out[1])


def lsm_price(option_type, strike, expiry, exercise, spot, rate, q, vol, num_paths, num_steps, seed, degree=2,
              dates=None, normals=None):
    out = np.zeros(2)
    d = None if dates is None else np.ascontiguousarray(dates, dtype=np.float64)
    z = None if normals is None else np.ascontiguousarray(normals, dtype=np.float64)
    st = lib().orc_lsm_price(option_type, strike, expiry, exercise, _ptr(d), 0 if d is None else len(d), spot,
                             rate, q, vol, num_paths, num_steps, seed, degree, _ptr(z), _ptr(out))
    if st != 0:
        raise RuntimeError(f"orc_lsm_price status {st}")
    return float(out[0]), float(out[1])


def sobol_points(dims, seed, count):
    out = np.zeros((count, dims))
    st = lib().orc_sobol_points(dims, seed & ((1 << 64) - 1), count, _ptr(out))
    if st != 0:
        raise RuntimeError(f"orc_sobol_points status {st}")
    return out


def sobol_dimension(dim, seed):
    v = (C.c_uint64 * 64)()
    s = C.c_uint64()
    lib().orc_sobol_dimension(dim, seed & ((1 << 64) - 1), v, C.byref(s))
    return list(v), s.value


def mc_european_qmc(option_type, spot, strike, rate, q, vol, expiry, n_paths, n_steps, seed=0):
    out = np.zeros(2)
    st = lib().orc_mc_european_qmc(option_type, spot, strike, rate, q, vol, expiry, n_paths, n_steps,
                                   seed & ((1 << 64) - 1), _ptr(out))
    if st != 0:
        raise RuntimeError(f"orc_mc_european_qmc status {st}")
    return float(out[0]), float(out[1])


def sampled_vol(strikes, expiries, vols, strike, expiry):
    k = np.ascontiguousarray(strikes, dtype=np.float64)
    t = np.ascontiguousarray(expiries, dtype=np.float64)
    v = np.ascontiguousarray(vols, dtype=np.float64)
    return lib().orc_sampled_vol(_ptr(k), len(k), _ptr(t), len(t), _ptr(v), strike, expiry)


def lsm_bermudan(option_type, expiry, schedule, spot, rate, q, num_paths, num_steps, seed, dynamics=0, vol=0.0,
                 lv=None, heston=None, degree=2, normals=None):
    """Bermudan LSM with the exercise boundary; schedule = [(t, K), ...];
    lv = (strikes, expiries, vols[expiry][strike]); heston = (kappa, theta, xi, rho, v0).
    Returns (price, stderr, [(time, strike, boundary or None, itm, exercised), ...])."""
    ts = np.ascontiguousarray([a for a, _ in schedule], dtype=np.float64)
    ks = np.ascontiguousarray([b for _, b in schedule], dtype=np.float64)
    lk = lt = lvv = None
    if lv is not None:
        lk = np.ascontiguousarray(lv[0], dtype=np.float64)
        lt = np.ascontiguousarray(lv[1], dtype=np.float64)
        lvv = np.ascontiguousarray(lv[2], dtype=np.float64)
    h = heston or (0.0, 0.0, 0.0, 0.0, 0.0)
    z = None if normals is None else np.ascontiguousarray(normals, dtype=np.float64)
    out = np.zeros(2)
    bnd = np.zeros(5 * (len(schedule) + 1))
    nb = I64()
    st = lib().orc_lsm_bermudan(option_type, expiry, _ptr(ts), _ptr(ks), len(ts), dynamics, spot, rate, q, vol,
                                _ptr(lk), 0 if lk is None else len(lk), _ptr(lt), 0 if lt is None else len(lt),
                                _ptr(lvv), *h, num_paths, num_steps, seed, degree, _ptr(z), _ptr(out), _ptr(bnd),
                                C.byref(nb))
    if st != 0:
        raise RuntimeError(f"orc_lsm_bermudan status {st}")
    recs = []
    for i in range(nb.value):
        t, k, b, itm, ex = bnd[5 * i:5 * i + 5]
        recs.append((float(t), float(k), None if np.isnan(b) else float(b), int(itm), int(ex)))
    return float(out[0]), float(out[1]), recs


def wgsl_european(spot, strike, rate, vol, expiry, num_paths, num_steps, seed, is_call=True):
    p, s = D(), D()
    st = lib().orc_wgsl_european(spot, strike, rate, vol, expiry, num_paths, num_steps, seed, int(is_call),
                                 C.byref(p), C.byref(s))
    if st != 0:
        raise RuntimeError(f"orc_wgsl_european status {st}")
    return p.value, s.value


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)
