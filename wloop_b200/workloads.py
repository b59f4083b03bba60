"""The measurement workloads: synthetic gauge fields with the shapes, sizes and
parameter values of the five benchmark configurations (no real openQCD
configurations exist here; fields come from the seeded Philox generator).

  c1  8^4 periodic, eps 0.3, HYP2 + APE 0.5, nss 0 5 5 5, r,t <= 4   (seed 1)
  c2  24^3x48 open bc, eps 0.25, nss 0 10 10 10 10, r<=12, t<=16     (seed 2)
  c3  32^3x64 periodic, eps 0.2, nss 0 10 10 10 10 10, r<=16, t<=24  (seed 3)
  c4  batch: 48 x 16^3x32 + 16 x 24^3x48, eps ~ U[0.15,0.35],
      HYP2 + 4 APE levels (nss 0 5 5 5), r,t <= Ns/2                 (seed 1000+i)
  c5  serving: volumes from {16^3x32, 24^3x48, 32^3x64, 48^3x96},
      eps ~ U[0.15,0.35], bc open/periodic 50/50, Poisson arrivals   (seed 5000)

HYP2 means hyp_links alpha = (1.0, 1.0, 0.5) on all four directions with
projection, proj_iter = 4 (main/ms10.in:25); nss is incremental
(modules/wloop/smear.c:109-120), so "0,5,10,15 sweeps" is nss = 0 5 5 5.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Tuple

from .api import APE, WloopParms, aux_uniform

HYP2 = (1.0, 1.0, 0.5)
PROJ_ITER = 4


@dataclass
class Workload:
    name: str
    n: Tuple[int, int, int, int]
    bc: int
    eps: float
    seed: int
    parms: WloopParms

    @property
    def volume(self) -> int:
        return self.n[0] * self.n[1] * self.n[2] * self.n[3]


def parms(msl, nss, mwlt, mwlr) -> WloopParms:
    return WloopParms(msl=msl, nss=list(nss), mwlt=mwlt, mwlr=mwlr, op_smear=APE,
                      alpha_action=HYP2, alpha_ape=0.5, alpha_hyp=(0.0, 0.0),
                      proj_iter=PROJ_ITER)


C1 = Workload("c1_8^4_periodic", (8, 8, 8, 8), 3, 0.3, 1, parms(4, [0, 5, 5, 5], 4, 4))
C2 = Workload("c2_24^3x48_open", (48, 24, 24, 24), 0, 0.25, 2,
              parms(5, [0, 10, 10, 10, 10], 16, 12))
C3 = Workload("c3_32^3x64_periodic", (64, 32, 32, 32), 3, 0.2, 3,
              parms(6, [0, 10, 10, 10, 10, 10], 24, 16))


def batch_workloads() -> List[Workload]:
    """c4: 48 configurations of 16^3x32 then 16 of 24^3x48, r,t <= Ns/2."""
    out = []
    for i in range(64):
        ns, nt = (16, 32) if i < 48 else (24, 48)
        eps = 0.15 + 0.2 * aux_uniform(1000 + i, 0, 1)
        out.append(Workload(f"c4_{i}", (nt, ns, ns, ns), 3, eps, 1000 + i,
                            parms(4, [0, 5, 5, 5], ns // 2, ns // 2)))
    return out


SERVE_VOLUMES = [(32, 16, 16, 16), (48, 24, 24, 24), (64, 32, 32, 32), (96, 48, 48, 48)]


def serving_request(i: int, seed: int = 5000) -> Workload:
    """c5 request i: volume, eps and bc drawn from the seeded stream."""
    v = SERVE_VOLUMES[int(4 * aux_uniform(seed, i, 2)) % 4]
    eps = 0.15 + 0.2 * aux_uniform(seed, i, 3)
    bc = 0 if aux_uniform(seed, i, 4) < 0.5 else 3
    ns = v[1]
    return Workload(f"c5_{i}", v, bc, eps, seed * 100000 + i, parms(4, [0, 5, 5, 5], ns // 2, ns // 2))


def flops_per_config(w: Workload) -> dict:
    """Algorithmic flops (M = 198 per 3x3 complex product, piter = proj_iter)."""
    M = 198
    p = w.parms
    pit = p.proj_iter
    proj = 76 + 531 * pit
    V = w.volume
    hyp = (48 * 828 + 28 * proj) * V
    ape = (6 * 828 + 3 * proj) * V * sum(p.nss[:p.msl])
    contract = 0
    lines = 0
    for r in range(1, p.mwlr + 1):
        contract += 3 * p.mwlt * (2 * p.msl * M + 36 * p.msl ** 2) * V
        if r >= 2:
            lines += 3 * p.msl * M * V
    plaq = 2592 * V * p.msl
    return {"hyp": hyp, "ape": ape, "lines": lines, "contract": contract, "plaq": plaq,
            "total": hyp + ape + lines + contract}
