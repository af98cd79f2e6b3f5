"""Extract the Slater-determinant known-answer vectors from the reference's unit test.

Reads tests/test_sdet_ops.cpp of the SAFIRE source tree as text (it is never compiled or
run) and writes ``sdet_kats.json`` beside this script.  The values pinned there are:

  ov_base, ov2_base            log-overlaps           test_sdet_ops.cpp:70-71
  m_a (3x4), m_b (4x3)          A = PsiT, B = walker   test_sdet_ops.cpp:82-91
  v_ref, vc_ref, v_ref_2, vc_ref_2  full/compact G     test_sdet_ops.cpp:147-170
  inv_m_a, inv_ref, logdetA_ref inverse_logdet        test_sdet_ops.cpp:334-356
  ma_lu, mb_lu, xv_ref, ovlp_lu_ref  LUsolve          test_sdet_ops.cpp:358-389

Usage: python tests/golden/make_sdet_kats.py [path/to/test_sdet_ops.cpp]
"""
import json
import os
import re
import sys

# tests/test_sdet_ops.cpp under the SAFIRE source tree named by SAFIRE_REFERENCE_ROOT
SRC_DEFAULT = (os.path.join(os.environ["SAFIRE_REFERENCE_ROOT"], "tests", "test_sdet_ops.cpp")
               if os.environ.get("SAFIRE_REFERENCE_ROOT") else "")
NUM = r"[-+]?\s*\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"
CPLX = re.compile(rf"({NUM})\s*([-+])\s*(\d+(?:\.\d*)?(?:[eE][-+]?\d+)?)i")


def _numbers(body):
    out = []
    for m in CPLX.finditer(body):
        re_ = float(m.group(1).replace(" ", ""))
        im = float(m.group(3)) * (-1.0 if m.group(2) == "-" else 1.0)
        out.append([re_, im])
    return out


def _array(text, name, occurrence=0):
    pat = re.compile(r"nda::array<Type,\s*2>\s+" + re.escape(name) + r"\s*=\s*\{(.*?)\};", re.S)
    ms = list(pat.finditer(text))
    body = ms[occurrence].group(1)
    rows = re.findall(r"\{([^{}]*)\}", body)
    return [_numbers(r) for r in rows]


def _scalar_log(text, name):
    m = re.search(re.escape(name) + r"\s*=\s*std::log\(([^)]*)\)", text)
    return _numbers(m.group(1))[0]


def _scalar_type(text, name):
    m = re.search(re.escape(name) + r"\(nwalk,\s*Type\(([^)]*)\)\)", text)
    return _numbers(m.group(1))[0]


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else SRC_DEFAULT
    if not src or not os.path.isfile(src):
        sys.exit("usage: make_sdet_kats.py <path/to/test_sdet_ops.cpp> (or set SAFIRE_REFERENCE_ROOT)")
    text = open(src).read()
    kats = {
        "source": "tests/test_sdet_ops.cpp (SAFIRE)",
        "nwalk": 5,
        "ov_base_log_of": _scalar_log(text, "ov_base "),
        "ov2_base_log_of": _scalar_log(text, "ov2_base"),
        "m_a": _array(text, "m_a", 0),
        "m_b": _array(text, "m_b", 0),
        "v_ref": _array(text, "v_ref", 0),
        "vc_ref": _array(text, "vc_ref", 0),
        "v_ref_2": _array(text, "v_ref_2", 0),
        "vc_ref_2": _array(text, "vc_ref_2", 0),
        "inv_m_a": _array(text, "m_a", 1),
        "inv_ref": _array(text, "inv_ref", 0),
        "logdetA_ref": _scalar_type(text, "logdetA_ref"),
        "ma_lu": _array(text, "ma_lu", 0),
        "mb_lu": _array(text, "mb_lu", 0),
        "xv_ref": _array(text, "xv_ref", 0),
        "ovlp_lu_ref": _scalar_type(text, "ovlp_ref"),
    }
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sdet_kats.json")
    with open(out, "w") as f:
        json.dump(kats, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
