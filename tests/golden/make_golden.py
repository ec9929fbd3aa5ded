"""Extract the reference's golden vectors and known answers into a fixture.

Reads the shrinkers crate's own test modules AS TEXT (the crate itself
cannot be compiled here: no Rust toolchain) and writes
``reference_vectors.json`` next to this script.  Run it where the
reference checkout is available:

    python tests/golden/make_golden.py /path/to/shrinkers

Every entry records the file:line range it came from.  The JSON is
committed; tests never read the reference checkout at run time.
"""
from __future__ import annotations

import json
import os
import re
import sys


def _floats(block: str) -> list[float]:
    return [float(x.replace("_", "")) for x in re.findall(r"-?\d[\d_]*\.\d[\d_]*(?:e-?\d+)?", block)]


def _vec_after(text: str, name: str) -> list[float]:
    m = re.search(r"let %s: Vec<f64> = vec!\[(.*?)\];" % re.escape(name), text, re.S)
    if not m:
        raise SystemExit(f"golden vector {name} not found")
    return _floats(m.group(1))


def _line_of(text: str, needle: str) -> int:
    return text[: text.index(needle)].count("\n") + 1


def main(root: str) -> None:
    src = os.path.join(root, "src")
    out: dict = {}

    # ---- El Karoui golden master: src/deconvolution/mod.rs ----
    path = os.path.join(src, "deconvolution", "mod.rs")
    text = open(path).read()
    start = _line_of(text, "fn test_golden_master_regression")
    gm = text[text.index("fn test_golden_master_regression"):]
    gm = gm[: gm.index("// ── Convention tests")]
    evals = _floats(re.search(r"let evals = vec!\[(.*?)\];", gm, re.S).group(1))
    c = float(re.search(r"let c = ([\d.]+);", gm).group(1))
    n_points = int(re.search(r"let n_points = (\d+);", gm).group(1))
    eta = float(re.search(r"let eta = ([\d.]+);", gm).group(1))
    out["golden_master"] = {
        "source": f"src/deconvolution/mod.rs:{start}-{start + gm.count(chr(10))}",
        "evals": evals, "c": c, "n_points": n_points, "eta": eta, "method": "blocked",
        "epsilon": 1e-14,
        "density": _vec_after(gm, "expected_density"),
        "w_re": _vec_after(gm, "expected_w_re"),
        "sample_stieltjes_imag": _vec_after(gm, "expected_si"),
        "population_stieltjes_imag": _vec_after(gm, "expected_pi"),
    }

    # ---- known answer: convention A at z = 2 + 0.1i (mod.rs test_empirical_stieltjes_simple)
    i0 = text.index("fn test_empirical_stieltjes_simple")
    blk = text[i0: i0 + 1500]
    num = float(re.search(r"let expected_ga_imag = -([\d.]+)_f64 / 3\.0;", blk).group(1))
    out["empirical_at_point"] = {
        "source": f"src/deconvolution/mod.rs:{_line_of(text, 'fn test_empirical_stieltjes_simple')}",
        "evals": [1.0, 2.0, 3.0], "z": [2.0, 0.1], "ga_imag": -num / 3.0, "ga_real": 0.0,
    }

    # ---- term.rs known answer
    path = os.path.join(src, "stieltjes", "term.rs")
    text = open(path).read()
    ln = _line_of(text, "fn test_term_basic")
    m = re.search(r"stieltjes_term\(([\d.]+), ([\d.]+), ([\d.]+)\)", text[text.index("fn test_term_basic"):])
    out["term_basic"] = {"source": f"src/stieltjes/term.rs:{ln}",
                         "args": [float(m.group(1)), float(m.group(2)), float(m.group(3))],
                         "expected": [1.0 / 1.01, 0.1 / 1.01], "tol": 1e-15}

    # ---- cacheblock.rs: unsorted 7-value sym case, p = 1 case
    path = os.path.join(src, "stieltjes", "cacheblock.rs")
    text = open(path).read()
    i0 = text.index("fn test_symmetric_all_points_matches_reference")
    blk = text[i0: i0 + 3000]
    evals7 = _floats(re.search(r"let evals = vec!\[(.*?)\];", blk, re.S).group(1))
    eta7 = float(re.search(r"let eta = ([\d.]+);", blk).group(1))
    m1 = re.search(r"compute_all_stieltjes_blocked_tiled\(&\[([\d.]+)\], ([\d.]+)", blk)
    out["symmetric_small"] = {
        "source": f"src/stieltjes/cacheblock.rs:{_line_of(text, 'fn test_symmetric_all_points_matches_reference')}",
        "evals": evals7, "eta": eta7, "tol": 1e-12,
        "p1": {"lambda": float(m1.group(1)), "eta": float(m1.group(2)), "re": 0.0,
               "im": 1.0 / float(m1.group(2))},
        "big": {"n": 1000, "rule": "((i*7919) % 9973)/9973*4-2 sorted", "eta": 0.11, "tol": 1e-12},
    }

    # ---- estimation.rs: inverse BBP round trip and threshold
    path = os.path.join(src, "spiked", "estimation.rs")
    text = open(path).read()
    i0 = text.index("fn test_inverse_bbp_roundtrip")
    blk = text[i0: i0 + 800]
    ells = _floats(re.search(r"for ell in \[(.*?)\]", blk).group(1))
    gamma = float(re.search(r"let gamma = ([\d.]+);", blk).group(1))
    out["inverse_bbp_roundtrip"] = {
        "source": f"src/spiked/estimation.rs:{_line_of(text, 'fn test_inverse_bbp_roundtrip')}",
        "gamma": gamma, "sigma2": 1.0, "ells": ells, "tol": 1e-10,
    }
    out["bbp_threshold"] = {
        "source": f"src/spiked/estimation.rs:{_line_of(text, 'fn test_bbp_threshold_formula')}",
        "gamma": 0.25, "sigma2": 2.0, "expected": 4.5, "tol": 1e-12,
    }

    # ---- detection.rs: BEMA known counts
    path = os.path.join(src, "spiked", "detection.rs")
    text = open(path).read()
    out["bema_known"] = {
        "source": f"src/spiked/detection.rs:{_line_of(text, 'fn test_detect_spikes_bema_known')}",
        "bulk": {"n": 100, "start": 0.5, "step": 0.015}, "spikes": [5.0, 7.0, 10.0],
        "gamma": 0.25, "margin": 1.0, "k": 3,
    }
    out["bema_none"] = {
        "source": f"src/spiked/detection.rs:{_line_of(text, 'fn test_detect_spikes_bema_no_spikes')}",
        "bulk": {"n": 100, "start": 0.5, "step": 0.01}, "gamma": 0.25, "margin": 1.0, "k": 0,
    }
    out["mp_median_factor"] = {
        "source": f"src/spiked/detection.rs:{_line_of(text, 'fn test_mp_median_factor')}",
        "points": [[0.0, 1.0, 1e-3], [0.25, 0.916, 0.01], [1.0, 0.653, 0.01]],
    }

    # ---- nufft.rs: grid sizing pins
    path = os.path.join(src, "stieltjes", "nufft.rs")
    text = open(path).read()
    out["nufft_grid"] = {
        "source": f"src/stieltjes/nufft.rs:{_line_of(text, 'fn grid_size_is_capped_and_independent_of_p')}",
        "cases": [[4.0, 1e-4, 65536], [2.0, 0.01, 32768], [2.0, 1e-300, 65536]],
    }

    # ---- config.rs: auto-resolution pins
    path = os.path.join(src, "config.rs")
    text = open(path).read()
    i0 = text.index("fn test_auto_resolution_is_parallelism_aware")
    blk = text[i0: i0 + 3000]
    cases = []
    for par, p, meth in re.findall(
            r"Parallelism::(\w+),\s*([\d_]+)usize,\s*StieltjesMethod::(\w+)", blk):
        cases.append([par == "Parallel", int(p.replace("_", "")), meth])
    out["auto_resolution"] = {
        "source": f"src/config.rs:{_line_of(text, 'fn test_auto_resolution_is_parallelism_aware')}",
        "cases": cases,
    }

    # ---- inverse nonlinear shrinkage: QIS golden master (deconvolution/inverse.rs)
    path = os.path.join(src, "deconvolution", "inverse.rs")
    text = open(path).read()
    i0 = text.index("fn qis_golden_master")
    blk = text[i0: text.index("\n    }\n", i0)]
    sp = text[text.index("fn spectrum(p: usize)"):]
    sp = sp[: sp.index("}")]
    fl = _floats(sp)  # lambda_i = base + (i + 1.0) * step
    base, step = fl[0], fl[2]
    rows = re.findall(r"\((\d+),\s*(-?[\d_.e-]+),\s*(-?[\d_.e-]+)\)", blk)
    out["qis_golden"] = {
        "source": f"src/deconvolution/inverse.rs:{_line_of(text, 'fn qis_golden_master')}",
        "spectrum": {"base": base, "step": step,
                     "p": int(re.search(r"spectrum\((\d+)\)", blk).group(1))},
        "c": float(re.search(r"let c = ([\d.]+);", blk).group(1)),
        "smoothing": _floats(re.search(r"nls\.smoothing, ([\d_.]+)", blk).group(1))[0],
        "rows": [[int(i), float(t.replace("_", "")), float(w.replace("_", ""))]
                 for i, t, w in rows],
        "max_relative": 1e-11,
    }

    # ---- fft5 accuracy sweep: the reference's own measured output
    # (docs/pareto/order_sweep.jsonl, written by examples/measure_fft_order_sweep.rs
    # on benches/support/mod.rs:65-80 harness_spectrum, eta = 1/sqrt(p),
    # error = rel-L2 vs the exact sums, support/mod.rs:126-135).
    path = os.path.join(root, "docs", "pareto", "order_sweep.jsonl")
    rows = [json.loads(line) for line in open(path) if line.strip()]
    out["fft5_order_sweep"] = {
        "source": "docs/pareto/order_sweep.jsonl (examples/measure_fft_order_sweep.rs)",
        "printed_digits": 4,
        "rows": [{k: r[k] for k in ("kind", "p", "order", "m", "err", "pad_mult") if k in r}
                 for r in rows],
    }
    ex = os.path.join(src, "stieltjes", "fft5.rs")
    text = open(ex).read()
    out["fft5_pipeline_ordering"] = {
        "source": f"src/stieltjes/fft5.rs:{_line_of(text, 'fn test_heptic_default_not_worse_on_pipeline')}",
        "p": 5000, "c": 0.5, "m": 8192, "outliers": ["hi*2.3", "lo*0.35"],
        "bulk_rule": "lo + ((i+0.5)/p)*(hi-lo)", "inv_p": "1/p (p excludes the outliers)",
        "assert": "e_cubic < e_linear and e_heptic <= e_cubic",
    }

    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the shrinkers crate checkout>")
    main(sys.argv[1])
