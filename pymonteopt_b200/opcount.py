"""Frozen FP32 operation table of the transport algorithm (roofline numerator).

Counts are per event, for the arithmetic the restatement performs on REAL
values (oracle/vmc_oracle_body.h, which follows
pymopt/voxel_gpu/_cukernel.py:27-227): every add, subtract, multiply and
compare is one FP32 operation, a multiply feeding an add counts once (one
FFMA issue), and square roots, reciprocals, logarithms and sines/cosines are
counted separately as MUFU operations.  The integer Philox work (ten rounds of
two 32x32 multiplies per draw) is reported beside them, not in the FP32
numerator; a draw serves each interaction, and Fresnel decisions and
roulettes mostly take the interaction's spare uniform.

Event counts come from the kernel's own integer counters (interactions,
face crossings, Fresnel evaluations, reflections, roulette draws, photons), so
``fp32_ops(counters)`` is the algorithmic FP32 work of a launch.

Per event:

* interaction — step draw (u, log, scale: 2 + 1 MUFU), final face-distance
  pass (3 x (face - p, x 1/v), 3 compares, db*mu_t, st >= db*mu_t: 11), hop
  (st/mu_t, 3 FFMA: 4), absorption (2), roulette test (1), Henyey-Greenstein
  cos(theta) (6 + 1 MUFU), sin(theta) (3 + 1 MUFU), azimuth (5 + 2 MUFU),
  rotation (17 + 2 MUFU), renormalisation (6 + 1 MUFU), inverse direction
  (3 MUFU): 57 FP32 + 11 MUFU;
* crossing — face-distance pass (11), move to the face (3), optical depth
  update (1): 15 FP32;
* Fresnel evaluation — cosines, sines and the reflectance (26 + 4 MUFU);
* transmission through an index step — refracted direction, renormalisation
  and inverse direction (9 + 4 MUFU);
* reflection — mirrored direction component and its inverse (2);
* roulette draw — compare and weight update (2);
* photon — source set-up and exit tally (12 + 2 MUFU).
"""
from __future__ import annotations

from . import _abi as A

FP32 = {"interaction": 57, "crossing": 15, "fresnel": 26, "transmission": 9, "reflection": 2,
        "roulette": 2, "photon": 12}
MUFU = {"interaction": 11, "crossing": 0, "fresnel": 4, "transmission": 4, "reflection": 0,
        "roulette": 0, "photon": 2}
PHILOX_INT_OPS = 70          # integer instructions per Philox4x32-10 draw (10 rounds)


def event_counts(counters) -> dict:
    c = [int(x) for x in counters]
    fres = c[A.PMO_C_FRESNEL]
    refl = c[A.PMO_C_REFLECT]
    return {"interaction": c[A.PMO_C_INTERACT], "crossing": c[A.PMO_C_CROSS], "fresnel": fres,
            "transmission": max(fres - refl, 0), "reflection": refl,
            "roulette": c[A.PMO_C_ROULETTE], "photon": c[A.PMO_C_PHOTONS]}


def fp32_ops(counters) -> int:
    ev = event_counts(counters)
    return sum(FP32[k] * v for k, v in ev.items())


def mufu_ops(counters) -> int:
    ev = event_counts(counters)
    return sum(MUFU[k] * v for k, v in ev.items())


def philox_draws(counters) -> int:
    """One draw per interaction plus the extra draws of Fresnel decisions and
    roulettes that found the step's spare uniform taken."""
    c = [int(x) for x in counters]
    return c[A.PMO_C_INTERACT] + c[A.PMO_C_XDRAWS]
