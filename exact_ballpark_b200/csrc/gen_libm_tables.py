# SPDX-License-Identifier: LGPL-2.1-or-later
"""Writes ebb_libm_tables.h: glibc 2.34 aarch64's libm constants and tables as exact C++ literals.

The values are not typed here. They are read from the reference's own Python transcriptions of glibc's libm
(exact_ballpark/dlibm.py, vec_exp.py, vec_libm.py, dlibm_powf.py), which hold them as Python source, and printed as
hexadecimal floating literals (C++17; exact by construction) or as hexadecimal integers for the words that are bit
patterns. The header is committed; this script is only rerun when the transcriptions change:

    EXACT_BALLPARK_REF=<checkout of exact-ballpark> python exact_ballpark_b200/csrc/gen_libm_tables.py

The reference modules bind `math.fma` at import (Python 3.13); on an older interpreter an exact stand-in is
installed first (the constants do not depend on it).
"""

from __future__ import annotations

import math
import os
import struct
import sys
from fractions import Fraction
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "ebb_libm_tables.h"


def _exact_fma(a, b, c):
    a, b, c = float(a), float(b), float(c)
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)):
        return a * b + c
    v = Fraction(a) * Fraction(b) + Fraction(c)
    return float(v) if v != 0 else (a * b + c)


def _load():
    ref = os.environ.get("EXACT_BALLPARK_REF")
    if not ref:
        raise SystemExit("set EXACT_BALLPARK_REF to a checkout of exact-ballpark (the tables are read from its modules)")
    sys.path.insert(0, os.path.join(ref, "src"))
    if not hasattr(math, "fma"):
        math.fma = _exact_fma
    from exact_ballpark import dlibm, dlibm_powf, vec_exp, vec_libm
    return dlibm, vec_exp, vec_libm, dlibm_powf


def dlit(x: float) -> str:
    """A double as an exact C++ literal."""
    if math.isnan(x):
        raise ValueError("NaN in a table")
    if math.isinf(x):
        return "(-EBB_INF)" if x < 0 else "EBB_INF"
    h = float(x).hex()
    return h if not h.startswith("-") else "-" + h[1:]


def u64(x: int) -> str:
    return f"0x{x & 0xFFFFFFFFFFFFFFFF:016x}ULL"


def u32(x: int) -> str:
    return f"0x{x & 0xFFFFFFFF:08x}u"


def fbits(x: float) -> int:
    return struct.unpack("<I", struct.pack("<f", x))[0]


def main() -> None:
    dlibm, vec_exp, vec_libm, dlibm_powf = _load()
    lines = [
        "// SPDX-License-Identifier: LGPL-2.1-or-later",
        "// glibc 2.34 aarch64 libm constants and tables, generated by gen_libm_tables.py from the reference's",
        "// transcriptions (exact_ballpark/dlibm.py, vec_exp.py, vec_libm.py, dlibm_powf.py). Do not edit.",
        "// Doubles are hexadecimal floating literals (exact); bit-pattern words are hexadecimal integers.",
        "#pragma once",
        "",
    ]

    def scalar_d(prefix, mod, names):
        for n in names:
            lines.append(f"#define {prefix}_{n} ({dlit(getattr(mod, n))})")

    def scalar_i(prefix, mod, names):
        for n in names:
            lines.append(f"#define {prefix}_{n} {u64(getattr(mod, n))}")

    def table_d(name, values, per=4):
        vals = [dlit(v) for v in values]
        body = ",\n    ".join(", ".join(vals[i:i + per]) for i in range(0, len(vals), per))
        lines.append(f"#define {name}_N {len(vals)}")
        lines.append(f"#define {name}_INIT {{ \\\n    " + body.replace("\n", " \\\n") + " }")

    def table_u64(name, values, per=4):
        vals = [u64(v) for v in values]
        body = ",\n    ".join(", ".join(vals[i:i + per]) for i in range(0, len(vals), per))
        lines.append(f"#define {name}_N {len(vals)}")
        lines.append(f"#define {name}_INIT {{ \\\n    " + body.replace("\n", " \\\n") + " }")

    def table_u32(name, values, per=6):
        vals = [u32(v) for v in values]
        body = ",\n    ".join(", ".join(vals[i:i + per]) for i in range(0, len(vals), per))
        lines.append(f"#define {name}_N {len(vals)}")
        lines.append(f"#define {name}_INIT {{ \\\n    " + body.replace("\n", " \\\n") + " }")

    # ---- double sin, cos, sincos, branred, log (dlibm.py) ----
    lines.append("// ---- sin, cos, sincos, __branred, log (dlibm.py) ----")
    scalar_d("DL", dlibm, ["TAYLOR_LIMIT", "BIG", "TOINT", "S1", "S2", "S3", "S4", "S5", "CS2", "CS4", "CS6", "SN3",
                           "SN5", "HPINV", "MP1", "MP2", "PP3", "PP4", "HP0", "HP1", "BR_TM600", "BR_SPLIT", "BR_TM24",
                           "BR_BIG", "BR_BIG1", "BR_TOVERP0", "BR_HP0", "BR_MP1", "BR_MP2", "BR_HP1", "LOG_TWO27",
                           "LOG_TWO52", "LOG_LN2HI", "LOG_LN2LO"])
    scalar_i("DL", dlibm, ["K_TINY_SIN", "K_TINY_COS", "K_DO_SIN", "K_MID", "K_REDUCE", "K_HUGE", "BR_T576_HI",
                           "BR_EXP_LIMIT", "BR_EXP_BIAS", "LOG_NEG_LO", "LOG_RANGE", "LOG_NEG_OFF", "LOG_NEG_52"])
    table_d("DL_SINCOSTAB", dlibm.SINCOSTAB)
    table_d("DL_BR_TOVERP", dlibm.BR_TOVERP)
    table_d("DL_LOG_A", dlibm.LOG_A)
    table_d("DL_LOG_B", dlibm.LOG_B)
    table_d("DL_LOG_TAB", [v for pair in dlibm.LOG_TAB for v in pair])
    # ---- exp (vec_exp.py) ----
    lines.append("// ---- exp (vec_exp.py; __exp_data) ----")
    scalar_d("DX", vec_exp, ["INVLN2N", "NEGLN2HIN", "NEGLN2LON", "C2", "C3", "C4", "C5", "TWO_1009", "TWO_M1022"])
    table_u64("DX_TAB", vec_exp.TABLE)
    # ---- float functions and pow (vec_libm.py) ----
    lines.append("// ---- expf, logf, sinf, cosf, acosf, atanf, atan2f, pow (vec_libm.py) ----")
    L = vec_libm
    table_u64("FL_EXP2F_TAB", L.EXP2F_TAB)
    scalar_d("FL", L, ["EXPF_INVLN2", "LOGF_LN2", "HPI_INV", "HPI", "PI63", "POW_LN2HI", "POW_LN2LO"])
    table_d("FL_EXPF_C", L.EXPF_C)
    table_d("FL_LOGF_TAB", [v for pair in L.LOGF_TAB for v in pair])
    table_d("FL_LOGF_A", L.LOGF_A)
    table_d("FL_SINCOSF_SIGN", L.SINCOSF_SIGN)
    table_d("FL_COSF_C", L.COSF_C)
    table_d("FL_SINF_S", L.SINF_S)
    table_u32("FL_INV_PIO4", L.INV_PIO4)
    table_d("FL_ATANF_HI", L.ATANF_HI)
    table_d("FL_ATANF_LO", L.ATANF_LO)
    fnames = ["EXPF_OFLOW", "EXPF_UFLOW", "EXPF_MAY_UFLOW", "ACOSF_PS0", "ACOSF_PS1", "ACOSF_PS2", "ACOSF_PS3",
              "ACOSF_PS4", "ACOSF_PS5", "ACOSF_QS1", "ACOSF_QS2", "ACOSF_QS3", "ACOSF_QS4", "ACOSF_PI",
              "ACOSF_PIO2_HI", "ACOSF_PIO2_LO", "ACOSF_NEG_PIO2_LO", "ACOSF_TWO_PIO2_LO"] + \
             [f"ATANF_T{i}" for i in range(11)] + \
             ["ATANF_HUGE", "ATANF_HI3", "ATANF_LO3", "ATAN2F_PI", "ATAN2F_NEG_PI", "ATAN2F_TINY", "ATAN2F_NEG_TINY",
              "ATAN2F_PIO2", "ATAN2F_NEG_PIO2", "ATAN2F_PIO4", "ATAN2F_NEG_PIO4", "ATAN2F_NEG_PI_LO",
              "ATAN2F_NEG_HALF_PI_LO", "MAY_UFLOWF"]
    for n in fnames:
        lines.append(f"#define FL_{n}_BITS {u32(fbits(getattr(L, n)))}")
    lines.append(f"#define FL_POW_OFF {u64(L.POW_OFF)}")
    lines.append(f"#define FL_SIGN_BIAS {u64(L.SIGN_BIAS)}")
    table_d("FL_POW_A", L.POW_A)
    table_d("FL_POW_TAB", [v for row in L.POW_TAB for v in row], per=3)
    # ---- powf (dlibm_powf.py; __powf_log2_data, and __exp2f_data as expf's) ----
    lines.append("// ---- powf (dlibm_powf.py; __powf_log2_data; its exp2 table and cubic are expf's) ----")
    P = dlibm_powf
    if list(P.POWF_EXP2_TAB) != list(L.EXP2F_TAB) or list(P.POWF_EXP2_C) != list(L.EXPF_C):
        raise SystemExit("powf's exp2 table or cubic differs from expf's")
    table_d("FL_POWF_INVC", P.POWF_LOG2_INVC)
    table_d("FL_POWF_LOGC", P.POWF_LOG2_LOGC)
    table_d("FL_POWF_A", P.POWF_A)
    scalar_d("FL", P, ["POWF_OFLOW", "POWF_RND"])
    for n in ("POWF_UFLOW", "POWF_MAY_UFLOW"):
        lines.append(f"#define FL_{n}_BITS {u64(getattr(P, n))}")
    for n in ("POWF_TINY_F", "POWF_OFLOWF_X", "POWF_UFLOWF_X", "POWF_MAY_UFLOWF_X"):
        lines.append(f"#define FL_{n} {u32(getattr(P, n))}")
    OUT.write_text("\n".join(lines) + "\n")
    print(f"wrote {OUT} ({len(lines)} lines)")


if __name__ == "__main__":
    main()
