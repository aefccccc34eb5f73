"""The reference's own test workload, restated: spin-polarised electrons in a flat Landau level
on a 3 x 4 torus mesh (Nk = 12, Gk = (3, 4)), Ne = 4 (filling 1/3), with a screened Coulomb
interaction projected to the lowest Landau level and the magnetic-translation phases
(MomentumED/test/example1_FQH_Laughlin.jl:1-94).  H_two takes momentum COORDINATES (k / Gk as
exact fractions, or floats when a float kshift is given), so ED_scatterlist_twobody runs its
coordinate branch (MomentumED/src/preparation/scat_list.jl:442-497), the default path of that
test.  Test infrastructure: used by the parity tests only.

The arithmetic follows the Julia source operation for operation (x^2 as x*x, left-to-right
products, 0.5 * Rational converted to Float64 first); cispi is computed with an exact
reduction to a quarter turn so that integer and half-integer arguments give exact 0 and +-1.
"""
from __future__ import annotations

import math

import numpy as np

K_LIST = np.array([[0, 1, 2, 0, 1, 2, 0, 1, 2, 0, 1, 2],
                   [0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3]], np.int64)     # example1_FQH_Laughlin.jl:4-5
GK = (3, 4)
NE = 4
NEIGEN = 10                                                             # example1_FQH_Laughlin.jl:105

GL = math.sqrt(2.0 * math.pi / math.sqrt(0.75))     # magnetic length scale from the Brillouin zone area
D_L = 5.0                                            # screening length / magnetic length
W0 = 1.0                                             # interaction strength
G12_ANGLE = 2.0 * math.pi / 3.0                      # angle between the reciprocal vectors


def VFF(q1: float, q2: float) -> float:
    """W0 / |ql| tanh(|ql| D) exp(-q^2 l^2 / 2) on the triangular metric (W0 D at q = 0)."""
    ql = math.sqrt(q1 * q1 + q2 * q2 + 2.0 * math.cos(G12_ANGLE) * q1 * q2) * GL
    if ql == 0.0:
        return W0 * D_L
    return W0 / ql * math.tanh(ql * D_L) * math.exp(-0.5 * (ql * ql))


def ita(g1: int, g2: int) -> int:
    return 1 if (g1 % 2 == 0 and g2 % 2 == 0) else -1


def ql_cross(a1, a2, b1, b2):
    return a1 * b2 - a2 * b1


def cispi(x: float) -> complex:
    """exp(i pi x) with x reduced exactly to the nearest quarter turn."""
    r = math.fmod(x, 2.0)
    if r < 0.0:
        r += 2.0
    n = int(round(2.0 * r))
    f = r - 0.5 * n
    s, c = math.sin(math.pi * f), math.cos(math.pi * f)
    n %= 4
    cr, ci = ((c, s), (-s, c), (-c, -s), (s, -c))[n]
    return complex(cr + 0.0, ci + 0.0)


def _round_nearest(v) -> int:
    return int(round(v))          # ties to even, for floats and Fractions alike (RoundNearest)


def V_int(kf1, kf2, ki2, ki1, cf1=1, cf2=1, ci2=1, ci1=1) -> complex:
    """Two-body matrix element with the magnetic-translation phases, summed over reciprocal
    vectors with |g1|, |g2|, |g1 - g2| <= 2 (example1_FQH_Laughlin.jl:54-89)."""
    d = [ki1[i] - kf1[i] for i in range(2)]
    q = [d[i] - _round_nearest(d[i]) for i in range(2)]                     # rem(., 1, RoundNearest)
    gs1 = [_round_nearest(ki1[i] - kf1[i] - q[i]) for i in range(2)]
    gs2 = [_round_nearest(kf2[i] - ki2[i] - q[i]) for i in range(2)]
    vr, vi = 0.0, 0.0
    nshell = 2
    for g1 in range(-nshell, nshell + 1):
        for g2 in range(-nshell, nshell + 1):
            if abs(g1 - g2) > nshell:
                continue
            qq1 = q[0] + g1
            qq2 = q[1] + g2
            pa = 0.5 * ql_cross(ki1[0], ki1[1], kf1[0], kf1[1])
            pa += 0.5 * ql_cross(ki1[0] + kf1[0], ki1[1] + kf1[1], qq1, qq2)
            pa += 0.5 * ql_cross(ki2[0], ki2[1], kf2[0], kf2[1])
            pa += 0.5 * ql_cross(ki2[0] + kf2[0], ki2[1] + kf2[1], -qq1, -qq2)
            ph = cispi(2.0 * pa)
            sgn = ita(g1 + gs1[0], g2 + gs1[1]) * ita(g1 + gs2[0], g2 + gs2[1])
            v = VFF(float(qq1), float(qq2))
            vr += (sgn * ph.real) * v
            vi += (sgn * ph.imag) * v
    return complex(vr, vi)
