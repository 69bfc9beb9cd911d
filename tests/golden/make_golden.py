"""Extracts the reference's known-answer vectors for the Monte Carlo path into
small JSON fixtures next to this script.

Reads (once, in a container where the openferric source tree is mounted):
  tests/lsm_reference.rs                 Longstaff-Schwartz (2001) Table 1 cases
  tests/fixtures/heston_params.csv       QuantLib Heston (Lewis) parameters
  tests/fixtures/heston_expected_put_call.csv
  tests/fixtures/asian_arithmetic_cases4.csv
  tests/fang_oosterlee_heston.rs         Fang-Oosterlee (2008) parameter set and values
  tests/bermudan_quantlib.rs             QuantLib FD Bermudan cases and the LSM engine settings
The fixtures are committed so that the GPU tests need no access to the
reference tree.

    python tests/golden/make_golden.py --reference PATH
"""
import argparse
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))


def _num(expr: str) -> float:
    expr = expr.strip()
    if "/" in expr:
        a, b = expr.split("/")
        return float(a) / float(b)
    return float(expr)


def _csv_rows(path):
    rows = []
    header = None
    with open(path) as f:
        for line in f:
            t = line.strip()
            if not t or t.startswith("#"):
                continue
            parts = [p.strip() for p in t.split(",")]
            if header is None:
                header = parts
                continue
            rows.append(dict(zip(header, parts)))
    return rows


def lsm_table1(ref):
    src = open(os.path.join(ref, "tests/lsm_reference.rs")).read()
    body = src[src.index("fn longstaff_schwartz_table1_cases"):]
    body = body[:body.index("\n}\n")]
    cases = []
    for m in re.finditer(r"LsmAmericanPutCase\s*\{(.*?)\}", body, re.S):
        fields = dict(re.findall(r"(\w+):\s*([-0-9.eE_]+)", m.group(1)))
        cases.append({k: float(v.replace("_", "")) for k, v in fields.items()})
    test = src[src.index("fn test_lsm_longstaff_schwartz_table1_american_put"):]
    cfg = {}
    for name in ("num_paths", "num_steps", "seed"):
        mm = re.search(rf"let {name}\s*(?::\s*\w+)?\s*=\s*([0-9_]+)", test)
        if mm:
            cfg[name] = int(mm.group(1).replace("_", ""))
    mm = re.search(r"LongstaffSchwartzEngine::new\(([^)]*)\)", test)
    return {"source": "tests/lsm_reference.rs (Longstaff-Schwartz 2001, Table 1)", "strike": 40.0, "rate": 0.06,
            "dividend_yield": 0.0, "engine": cfg, "engine_call": mm.group(1) if mm else None, "cases": cases}


def heston_lewis(ref):
    p = _csv_rows(os.path.join(ref, "tests/fixtures/heston_params.csv"))[0]
    rows = _csv_rows(os.path.join(ref, "tests/fixtures/heston_expected_put_call.csv"))
    return {"source": "tests/fixtures/heston_params.csv, heston_expected_put_call.csv (QuantLib Lewis table)",
            "params": {k: float(v) for k, v in p.items()},
            "rows": [{"strike": float(r["strike"]), "put": float(r["expected_put"]), "call": float(r["expected_call"])}
                     for r in rows]}


def asian_cases4(ref):
    rows = _csv_rows(os.path.join(ref, "tests/fixtures/asian_arithmetic_cases4.csv"))
    out = []
    for r in rows:
        out.append({"line": int(r["source_line"]), "option_type": "Put" if "Put" in r["option_type"] else "Call",
                    "underlying": _num(r["underlying"]), "strike": _num(r["strike"]),
                    "dividend_yield": _num(r["dividend_yield"]), "risk_free_rate": _num(r["risk_free_rate"]),
                    "first": _num(r["first"]), "length": _num(r["length"]), "fixings": int(_num(r["fixings"])),
                    "volatility": _num(r["volatility"]), "control_variate": r["control_variate"] == "true",
                    "expected": _num(r["expected"])})
    return {"source": "tests/fixtures/asian_arithmetic_cases4.csv (QuantLib cases4)", "cases": out}


def fang_oosterlee(ref):
    src = open(os.path.join(ref, "tests/fang_oosterlee_heston.rs")).read()
    consts = {k: float(v) for k, v in re.findall(r"const (\w+): f64 = ([-0-9.eE]+);", src)}
    vals = []
    for m in re.finditer(r"fn fang_oosterlee_heston_t(\d+)_k(\d+)\(\)\s*\{(.*?)\n\}", src, re.S):
        ref_v = re.search(r"let reference = ([-0-9.eE]+);", m.group(3))
        tol = re.search(r"err < ([-0-9.eE]+)", m.group(3))
        if ref_v:
            vals.append({"maturity": float(m.group(1)), "strike": float(m.group(2)), "reference": float(ref_v.group(1)),
                         "tolerance": float(tol.group(1)) if tol else None})
    return {"source": "tests/fang_oosterlee_heston.rs (Fang-Oosterlee 2008)", "params": consts, "values": vals}


def bermudan_quantlib(ref):
    src = open(os.path.join(ref, "tests/bermudan_quantlib.rs")).read()
    grids = {}
    for name, body in re.findall(r"const (D\w+): &\[f64\] = &\[(.*?)\];", src, re.S):
        grids[name] = [float(x.replace("_", "")) for x in re.findall(r"[0-9][0-9_.eE]*", body)]
    fn = src[src.index("fn quantlib_reference_cases"):]
    fn = fn[:fn.index("\n}\n")]
    cases = []
    for m in re.finditer(r"QlBermudanCase\s*\{(.*?)\}", fn, re.S):
        f = dict(re.findall(r"(\w+):\s*([^,]+),", m.group(1)))
        cases.append({"option_type": "Put" if "Put" in f["option_type"] else "Call",
                      "spot": float(f["spot"].replace("_", "")), "strike": float(f["strike"].replace("_", "")),
                      "rate": float(f["rate"].replace("_", "")), "dividend": float(f["dividend"].replace("_", "")),
                      "vol": float(f["vol"].replace("_", "")), "expiry": float(f["expiry"].replace("_", "")),
                      "dates": grids[f["dates"].strip()],
                      "quantlib_fd_price": float(f["quantlib_fd_price"].replace("_", ""))})
    test = src[src.index("fn bermudan_lsm_matches_quantlib_fd_within_half_percent_on_reference_puts"):]
    mm = re.search(r"LongstaffSchwartzEngine::new\(([0-9_]+),\s*([0-9_]+),\s*([0-9_]+)\)", test)
    tol = re.search(r"err <= ([0-9.]+)", test)
    return {"source": "tests/bermudan_quantlib.rs (QuantLib 1.41 FdBlackScholesVanillaEngine(2000, 400) Bermudan "
                      "prices; LSM put check)",
            "lsm_engine": {"num_paths": int(mm.group(1).replace("_", "")), "num_steps": int(mm.group(2).replace("_", "")),
                           "seed": int(mm.group(3).replace("_", ""))},
            "rel_tolerance": float(tol.group(1)), "cases": cases}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of an openferric source tree")
    a = ap.parse_args()
    fixtures = {
        "lsm_table1.json": lsm_table1(a.reference),
        "heston_lewis.json": heston_lewis(a.reference),
        "asian_cases4.json": asian_cases4(a.reference),
        "fang_oosterlee.json": fang_oosterlee(a.reference),
        "bermudan_quantlib.json": bermudan_quantlib(a.reference),
    }
    for name, data in fixtures.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(data, f, indent=1)
        print(name, "written")


if __name__ == "__main__":
    main()
