"""The IPRINT = 1 unit-3 text of POT3 (pot/pot3.f:402-418), formatted in
Python from the oracle's PHAC and COEF with the reference's edit
descriptors: FORMAT(1P11E11.3) and FORMAT(20X,I5,' COEFS=',1P8E12.3,/,25X,
' PHASE=',0P8F12.2).  Test helper."""
import math


def _fit(s, w):
    return s.rjust(w) if len(s) <= w else "*" * w


def edit_e(v, w):
    """1PEw.3: d.dddE+xx, or d.ddd+xxx for exponents beyond two digits."""
    if math.isnan(v):
        return _fit("NaN", w)
    if math.isinf(v):
        return _fit("-Infinity" if v < 0 else "Infinity", w)
    mant, ex = ("%.3E" % v).split("E")
    return _fit(mant + ("E" + ex if len(ex) <= 3 else ex), w)


def edit_f(v, w):
    return _fit("%.2f" % v, w)


def report(phac_of_k, coef, J, K, L):
    """phac_of_k(K) gives PHAC(K); coef is COEF(J+2, K+2, L/2, 2) (0-based)."""
    out = ["PHAC(1:KMAX1):\n"]
    vals = [edit_e(phac_of_k(k), 11) for k in range(2, K + 2)]
    for i in range(0, len(vals), 11):
        out.append("".join(vals[i:i + 11]) + "\n")
    out.append("Fourier amplitudes and phases:\n")
    if L > 8:
        for j in range(2, J + 1):
            amp = "".join(edit_e(coef[j - 1, 1, m, 0], 12) for m in range(8))
            ph = "".join(edit_f(coef[j - 1, 1, m, 1], 12) for m in range(8))
            out.append(" " * 20 + "%5d" % j + " COEFS=" + amp + "\n")
            out.append(" " * 25 + " PHASE=" + ph + "\n")
    return "".join(out)


def check(text, ref, atol=1e-11):
    """Every line of `text` equals the reference text character for
    character, except the PHAC values, which are deviations 1 - PH/PHMAX of
    order 1e-10 .. 1e-3: rounding noise of PHI moves them by about PHI's
    relative error, so they are compared as numbers, within their printed
    precision (half a unit in the 4th digit) plus atol."""
    a, b = text.split("\n"), ref.split("\n")
    assert len(a) == len(b), (len(a), len(b))
    assert a[0] == b[0] == "PHAC(1:KMAX1):"
    i = 1
    while not b[i].startswith("Fourier"):
        assert len(a[i]) == len(b[i])
        for k in range(0, len(b[i]), 11):
            x, y = float(a[i][k:k + 11]), float(b[i][k:k + 11])
            assert abs(x - y) <= 5e-4 * abs(y) + atol, (i, k, a[i][k:k + 11], b[i][k:k + 11])
        i += 1
    assert a[i:] == b[i:]
