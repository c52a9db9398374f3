"""Extract the golden vectors that the reference pins its field/FFT code with.

The reference (pcrumley/spectral_rs) keeps its known-answer vectors inline in its
Rust unit tests.  This script reads those test sources *as text* (the Rust crate
cannot be compiled here) and writes them as JSON fixtures next to this file, so
that the test-suite never needs the reference tree at run time.

Sources (paths relative to the reference project):
  src/flds/field.rs   copy_to_spectral (:487-570), copy_to_spatial (:572-655),
                      ghost_deposit (:657-723), ghosts_update (:726-795),
                      binomial_filter (:798-1543)
  src/flds/fft_2d.rs  get_2d_input (:180-477), forward_fft (:479-547),
                      fft_1d_roundtrip (:550-600), forward_fft2d (:602-907)
  src/flds/wave_num.rs wave_nums_init (:50-943)
  src/lib.rs          build_test_sim (:219-244): 24x12 grid, dt 0.1, delta 5,
                      c 3, dens 2, gamma_inj 5, n_pass 4; E_TOL (:28-32)

Usage:  python tests/golden/extract_golden.py /path/to/spectral_rs  (the reference checkout; required)
"""
import json
import os
import re
import sys

NUM = r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"


def _fn_body(src, name):
    # test functions live in the `mod tests` block at the end of each file
    src = src[src.index("mod tests"):]
    m = re.search(r"fn\s+" + re.escape(name) + r"\s*\(", src)
    if not m:
        raise KeyError(name)
    i = src.index("{", m.end())
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[i:j + 1]
    raise ValueError("unbalanced " + name)


def _vec_after(body, lhs_regex):
    m = re.search(lhs_regex + r"(?:[^=\n]*=)?\s*vec!\[", body)
    if not m:
        raise KeyError(lhs_regex)
    start = m.end()
    depth = 1
    for j in range(start, len(body)):
        if body[j] == "[":
            depth += 1
        elif body[j] == "]":
            depth -= 1
            if depth == 0:
                return body[start:j]
    raise ValueError("unbalanced vec")


def _reals(text):
    return [float(x) for x in re.findall(NUM, text)]


def _complexes(text):
    out = []
    for a, b in re.findall(r"Complex::new\(\s*(" + NUM + r")\s*,\s*(" + NUM + r")\s*\)", text):
        out.append([float(a), float(b)])
    return out


def main(ref):
    field = open(os.path.join(ref, "src/flds/field.rs")).read()
    fft = open(os.path.join(ref, "src/flds/fft_2d.rs")).read()
    wn = open(os.path.join(ref, "src/flds/wave_num.rs")).read()
    g = {"test_sim": {"size_x": 24, "size_y": 12, "dt": 0.1, "delta": 5, "c": 3.0,
                      "dens": 2, "gamma_inj": 5.0, "n_pass": 4},
         "e_tol": {"f32": 1e-4, "f64": 1e-13}}
    b = _fn_body(field, "copy_to_spectral")
    g["copy_to_spectral"] = {"input": _reals(_vec_after(b, r"let input")),
                             "expected": _reals(_vec_after(b, r"let expected_output"))}
    b = _fn_body(field, "copy_to_spatial")
    g["copy_to_spatial"] = {"input": _reals(_vec_after(b, r"let input")),
                            "expected": _reals(_vec_after(b, r"let expected_output"))}
    b = _fn_body(field, "ghost_deposit")
    g["ghost_deposit"] = {"input": _reals(_vec_after(b, r"let input")),
                          "expected": _reals(_vec_after(b, r"let expected_output"))}
    b = _fn_body(field, "ghosts_update")
    g["ghosts_update"] = {"input": _reals(_vec_after(b, r"let input")),
                          "expected": _reals(_vec_after(b, r"let expected_output"))}
    b = _fn_body(field, "binomial_filter")
    g["binomial_filter"] = {"input": _reals(_vec_after(b, r"let input")),
                            "expected": _reals(_vec_after(b, r"expected_out\.spatial")),
                            "n_pass": 4}
    b = _fn_body(fft, "get_2d_input")
    g["fft2d_input"] = _complexes(_vec_after(b, r"let input"))
    b = _fn_body(fft, "forward_fft2d")
    g["forward_fft2d"] = {"expected": _complexes(_vec_after(b, r"let out"))}
    b = _fn_body(fft, "forward_fft")
    g["forward_fft"] = {"input": _complexes(_vec_after(b, r"let mut input")),
                        "expected": _complexes(_vec_after(b, r"let out"))}
    b = _fn_body(fft, "fft_1d_roundtrip")
    g["fft_1d_roundtrip"] = {"input": _complexes(_vec_after(b, r"let mut input"))}
    b = _fn_body(wn, "wave_nums_init")
    g["wave_nums_init"] = {"k_x": _reals(_vec_after(b, r"k_x:")),
                           "k_y": _reals(_vec_after(b, r"k_y:")),
                           "k_norm": _reals(_vec_after(b, r"k_norm:"))}
    # shape checks: 26x14 ghosted, 24x12 interior
    assert len(g["copy_to_spectral"]["input"]) == 26 * 14
    assert len(g["copy_to_spectral"]["expected"]) == 24 * 12
    assert len(g["copy_to_spatial"]["input"]) == 24 * 12
    assert len(g["copy_to_spatial"]["expected"]) == 26 * 14
    for k in ("ghost_deposit", "ghosts_update", "binomial_filter"):
        assert len(g[k]["input"]) == 26 * 14, k
        assert len(g[k]["expected"]) == 26 * 14, k
    assert len(g["fft2d_input"]) == 24 * 12
    assert len(g["forward_fft2d"]["expected"]) == 24 * 12
    assert len(g["forward_fft"]["input"]) == 24 and len(g["forward_fft"]["expected"]) == 24
    for k in ("k_x", "k_y", "k_norm"):
        assert len(g["wave_nums_init"][k]) == 24 * 12, k
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")
    with open(out, "w") as f:
        json.dump(g, f, separators=(",", ":"))
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_golden.py /path/to/spectral_rs")
    main(sys.argv[1])
