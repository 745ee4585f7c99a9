"""Writes ref_log_table.inc: the reduction table of the float log that
precision mode 3 uses (ref_logf in common.cuh, og_log_f32 in the oracle).

For a float x = m * 2^e with m in [sqrt(1/2), sqrt(2)), k = round(128 (m - 1))
lies in [-38, 54].  Entry k holds r_k = round(1024 / (1 + k/128)) / 1024 (11
significant bits, so m * r_k and m * r_k - 1 are exact in double) and
L_k = -log(r_k) rounded to the nearest double (computed here with 50
significant digits).  Then log x = e ln 2 + L_k + log1p(m r_k - 1), with
|m r_k - 1| < 0.0066.

Run:  python usap_b200/csrc/ref_log_table.py  (rewrites the .inc beside it)
"""
import decimal
import os

K_MIN, K_MAX = -38, 54


def entries():
    decimal.getcontext().prec = 50
    out = []
    for k in range(K_MIN, K_MAX + 1):
        R = (2 * 131072 + (128 + k)) // (2 * (128 + k))   # round(131072 / (128 + k))
        r = decimal.Decimal(R) / decimal.Decimal(1024)
        L = -r.ln()
        out.append((R / 1024.0, float(str(L)) + 0.0))   # + 0.0: no negative zero
    return out


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    lines = ["/* generated by ref_log_table.py: {r_k, -log(r_k)} for k = %d..%d */" % (K_MIN, K_MAX)]
    for r, L in entries():
        lines.append("{%s, %s}," % (float.hex(r), float.hex(L)))
    with open(os.path.join(here, "ref_log_table.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
