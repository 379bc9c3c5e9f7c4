"""Pure-Python, line-by-line transliteration of Native_Mod's Cg / Bicg.

TEST INFRASTRUCTURE ONLY, small cases only (plain Python loops).  It is a
second, independent restatement used to pin the C++ oracle: on the same
inputs the two must agree bit for bit (Python floats are IEEE doubles and
every expression below is evaluated in the Fortran source's order, with no
FMA).  Each function cites the lines it follows, paths inside the T-Flows
tree (Sources/Process/Cpu/Native_Mod/...).

Arrays use Fortran 1-based indexing through a leading dummy element.
"""
import math

TINY = 1.0e-15   # Shared/Const_Mod.f90
HUGE = 1.0e+15


def _f(a):
    """0-based sequence -> 1-based list (index 0 unused)."""
    return [None] + [float(v) for v in a]


def _i(a):
    return [None] + [int(v) for v in a]


def nrms(ni, r, a_val, a_dia, x, norm):
    """Normalized_Root_Mean_Square.f90:33-63."""
    rms = 0.0
    for i in range(1, ni + 1):
        rms = rms + (r[i] * r[i]) / (a_val[a_dia[i]] * a_val[a_dia[i]])
    rms = math.sqrt(rms)
    if norm is None:
        x_min, x_max = +HUGE, -HUGE
        for i in range(1, ni + 1):
            x_min = x[i] if x[i] < x_min else x_min
            x_max = x[i] if x[i] > x_max else x_max
    else:
        x_min, x_max = 0.0, norm
    x_max_min = x_max - x_min
    x_max_min = TINY if TINY > x_max_min else x_max_min
    return rms / x_max_min


def solve(solver, prec, row, col, dia, val, x, b, miter, tol, norm=None):
    """Cg.f90:2-257 and Bicg.f90:2-269 with Prec_Form and Prec_Solve
    (jacobi, icc, none).  Returns (x, val, b, niter, fin_res) as
    0-based lists."""
    a_row, a_col, a_dia = _i(row), _i(col), _i(dia)
    a_val, x, b = _f(val), _f(x), _f(b)
    nt = len(row) - 1
    ni = nt
    bicg = solver == "bicg"
    z = [0.0] * (nt + 1)
    p1, q1, r1 = z[:], z[:], z[:]
    p2, q2, r2 = z[:], z[:], z[:]
    d, d_inv = z[:], z[:]
    res = 0.0
    # Normalize the system (Cg.f90:62-84)
    sum_a, sum_n = 0.0, 0
    for i in range(1, ni + 1):
        sum_a = sum_a + a_val[a_dia[i]]
        sum_n = sum_n + 1
    sum_a = sum_a / sum_n
    fn = 1.0 / sum_a
    for i in range(1, nt + 1):
        for j in range(a_row[i], a_row[i + 1]):
            a_val[j] = a_val[j] * fn
        b[i] = b[i] * fn
    # Prec_Form.f90:47-89
    if prec == "icc":
        for i in range(1, ni + 1):
            sm = a_val[a_dia[i]]
            for j in range(a_row[i] + 1, a_row[i + 1]):
                k = a_col[j]
                if k > i:
                    break
                sm = sm - d[k] * a_val[j] * a_val[j]
            d_inv[i] = sm
            d[i] = 1.0 / sm
    else:
        for i in range(1, ni + 1):
            if prec == "jacobi":
                d[i] = a_val[a_dia[i]]
                d_inv[i] = 1.0 / d[i]
            else:
                d[i] = 1.0

    def prec_solve(out, inp):   # Prec_Solve.f90:44-102
        if prec == "icc":
            for i in range(1, ni + 1):                       # forward
                sm = inp[i]
                for j in range(a_row[i] + 1, a_row[i + 1]):
                    k = a_col[j]
                    if k > i:
                        break
                    sm = sm - a_val[j] * out[k]
                out[i] = sm * d[i]
            for i in range(1, ni + 1):
                out[i] = out[i] * d_inv[i]
            for i in range(ni, 0, -1):                       # backward
                sm = out[i]
                for j in range(a_row[i + 1] - 1, a_row[i], -1):
                    k = a_col[j]
                    if k < i:
                        break
                    if k <= ni:
                        sm = sm - a_val[j] * out[k]
                out[i] = sm * d[i]
            return
        for i in range(1, ni + 1):
            out[i] = inp[i] * d_inv[i] if prec == "jacobi" else inp[i]

    bnrm2 = nrms(ni, b, a_val, a_dia, x, norm)
    it = 0
    if bnrm2 < tol:
        it = 0
    else:
        for i in range(1, ni + 1):           # Residual_Vector.f90:35-41
            r1[i] = b[i]
            for j in range(a_row[i], a_row[i + 1]):
                r1[i] = r1[i] - a_val[j] * x[a_col[j]]
        res = nrms(ni, r1, a_val, a_dia, x, norm)
        if res < tol:
            it = 0
        else:
            for i in range(1, ni + 1):
                if bicg:
                    r2[i] = r1[i]
                else:
                    p1[i] = r1[i]
            converged = False
            rho_old = 0.0
            for it in range(1, miter + 1):
                prec_solve(q1, r1)
                if bicg:
                    prec_solve(q2, r2)
                rho = 0.0
                for i in range(1, ni + 1):
                    rho = rho + q1[i] * (r2[i] if bicg else r1[i])
                if it == 1:
                    for i in range(1, ni + 1):
                        p1[i] = q1[i]
                        if bicg:
                            p2[i] = q2[i]
                else:
                    beta = rho / rho_old
                    for i in range(1, ni + 1):
                        p1[i] = q1[i] + beta * p1[i]
                        if bicg:
                            p2[i] = q2[i] + beta * p2[i]
                for i in range(1, ni + 1):
                    q1[i] = 0.0
                    if bicg:
                        q2[i] = 0.0
                    for j in range(a_row[i], a_row[i + 1]):
                        k = a_col[j]
                        q1[i] = q1[i] + a_val[j] * p1[k]
                        if bicg:
                            q2[i] = q2[i] + a_val[j] * p2[k]
                alfa = 0.0
                for i in range(1, ni + 1):
                    alfa = alfa + (p2[i] if bicg else p1[i]) * q1[i]
                alfa = rho / alfa
                for i in range(1, ni + 1):
                    x[i] = x[i] + alfa * p1[i]
                    r1[i] = r1[i] - alfa * q1[i]
                    if bicg:
                        r2[i] = r2[i] - alfa * q2[i]
                res = nrms(ni, r1, a_val, a_dia, x, norm)
                if res < tol:
                    converged = True
                    break
                rho_old = rho
            if not converged:
                it = miter   # Cg.f90:228 (do variable ends at miter+1)
    for i in range(1, nt + 1):                 # Cg.f90:245-250
        for j in range(a_row[i], a_row[i + 1]):
            a_val[j] = a_val[j] / fn
        b[i] = b[i] / fn
    return x[1:], a_val[1:], b[1:], it, res
