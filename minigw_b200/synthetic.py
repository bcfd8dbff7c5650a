"""Seeded synthetic G0W0 inputs with the benchmark shapes (no dataset is involved).

Recipe (one definition, used by the tests, the benchmark and the reference arm):
  rng = numpy.random.default_rng(seed)
  mo_energy: nocc occupied values sorted from U[-1.2, -0.3] Ha, then nvir virtual values
             sorted from U[0.05, 3.0] Ha; fermi_energy = (HOMO + LUMO) / 2.
  L[K, p, q] = N(0,1) * 0.3 * exp(-|p-q|/8) for K < 2*nmo, drawn on p <= q and mirrored
             (symmetric in p, q).
  eri_mo[p,q,r,s] = sum_K L[K,p,q] L[K,r,s], symmetrised over (pq) <-> (rs) so that the
             8-fold symmetry holds bit for bit; float64, C order.  The (ov|ov) block is a
             Gram matrix, hence PSD like a Coulomb metric.
  vxc_mo: symmetric, diagonal U[-0.6, -0.2], off-diagonal N(0, 0.01).

Named workloads (nmo, nocc, nfreq, npade, states):
  cfg1  "H2O-shaped":   24,  5, 200, 16, [4]                  (state 5, 1-based)
  cfg2  "mixed-vs-fp64": 120, 20,  64, 16, HOMO-2..LUMO+2
  cfg3  "large":        200, 30, 128, 16, HOMO-4..LUMO+4
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .gw_input import GwInput


@dataclass(frozen=True)
class Workload:
    name: str
    nmo: int
    nocc: int
    nfreq: int
    npade: int
    states: tuple[int, ...]

    @property
    def nph(self) -> int:
        return self.nocc * (self.nmo - self.nocc)

    @property
    def ncols(self) -> int:
        return len(self.states) * self.nmo

    def flops_per_frequency(self) -> float:
        n, m = float(self.nph), float(self.ncols)
        return n ** 3 / 3.0 + n * n * m + 3.0 * n * m


def around_gap(nocc: int, below: int, above: int) -> tuple[int, ...]:
    """0-based states HOMO-below .. LUMO+above (HOMO = nocc-1, LUMO = nocc)."""
    return tuple(range(nocc - 1 - below, nocc + above + 1))


WORKLOADS = {
    "cfg1": Workload("cfg1", 24, 5, 200, 16, (4,)),
    "cfg2": Workload("cfg2", 120, 20, 64, 16, around_gap(20, 2, 2)),
    "cfg3": Workload("cfg3", 200, 30, 128, 16, around_gap(30, 4, 4)),
}


def make_input(nmo: int, nocc: int, seed: int = 0, out_eri: np.ndarray | None = None) -> GwInput:
    """Generate one synthetic system (see the module docstring).  `out_eri` may be a
    preallocated (e.g. pinned) float64 buffer of nmo**4 elements to fill in place."""
    if not (0 < nocc < nmo):
        raise ValueError("need 0 < nocc < nmo")
    rng = np.random.default_rng(seed)
    nvir = nmo - nocc
    occ = np.sort(rng.uniform(-1.2, -0.3, nocc))
    vir = np.sort(rng.uniform(0.05, 3.0, nvir))
    mo = np.concatenate([occ, vir])
    fermi = 0.5 * (occ[-1] + vir[0])
    nk = 2 * nmo
    idx = np.arange(nmo)
    decay = 0.3 * np.exp(-np.abs(idx[:, None] - idx[None, :]) / 8.0)
    g = rng.standard_normal((nk, nmo, nmo))
    upper = np.triu(g)
    lfac = (upper + np.transpose(np.triu(g, 1), (0, 2, 1))) * decay
    lmat = lfac.reshape(nk, nmo * nmo)
    npq = nmo * nmo
    eri = out_eri.reshape(npq, npq) if out_eri is not None else np.empty((npq, npq))
    np.matmul(lmat.T, lmat, out=eri)
    # exact (pq)<->(rs) symmetry, blockwise to bound temporary memory
    blk = 2048
    for i0 in range(0, npq, blk):
        i1 = min(npq, i0 + blk)
        for j0 in range(i0, npq, blk):
            j1 = min(npq, j0 + blk)
            a = eri[i0:i1, j0:j1]
            b = eri[j0:j1, i0:i1].T
            s = 0.5 * (a + b)
            eri[i0:i1, j0:j1] = s
            eri[j0:j1, i0:i1] = s.T
    vxc = rng.normal(0.0, 0.01, (nmo, nmo))
    vxc = np.triu(vxc, 1)
    vxc = vxc + vxc.T
    vxc[idx, idx] = rng.uniform(-0.6, -0.2, nmo)
    return GwInput(eri_mo=eri.reshape(nmo, nmo, nmo, nmo), mo_energy=mo, vxc_mo=vxc, nocc=nocc,
                   fermi_energy=float(fermi))


def make_workload_input(w: Workload, seed: int = 0, out_eri: np.ndarray | None = None) -> GwInput:
    return make_input(w.nmo, w.nocc, seed, out_eri)


def make_input_on_device(nmo: int, nocc: int, seed: int = 0, device: int = 0, pin: bool = True) -> GwInput:
    """Same recipe as make_input (identical random draws), with the nmo^2 x nmo^2 ERI product and
    its symmetrisation done by torch on the GPU (FP64), then copied to (pinned) host memory.
    Only the rounding of the ERI sum differs from the numpy path.  Used for the large benchmark
    workloads, where the host GEMM would take minutes."""
    import torch

    rng = np.random.default_rng(seed)
    nvir = nmo - nocc
    occ = np.sort(rng.uniform(-1.2, -0.3, nocc))
    vir = np.sort(rng.uniform(0.05, 3.0, nvir))
    mo = np.concatenate([occ, vir])
    fermi = 0.5 * (occ[-1] + vir[0])
    nk = 2 * nmo
    idx = np.arange(nmo)
    decay = 0.3 * np.exp(-np.abs(idx[:, None] - idx[None, :]) / 8.0)
    g = rng.standard_normal((nk, nmo, nmo))
    lfac = (np.triu(g) + np.transpose(np.triu(g, 1), (0, 2, 1))) * decay
    npq = nmo * nmo
    dev = torch.device("cuda", device)
    lmat = torch.from_numpy(np.ascontiguousarray(lfac.reshape(nk, npq))).to(dev)
    e = lmat.t() @ lmat
    del lmat
    blk = 4096
    for i0 in range(0, npq, blk):
        i1 = min(npq, i0 + blk)
        for j0 in range(i0, npq, blk):
            j1 = min(npq, j0 + blk)
            s = 0.5 * (e[i0:i1, j0:j1] + e[j0:j1, i0:i1].t())
            e[i0:i1, j0:j1] = s
            e[j0:j1, i0:i1] = s.t()
    host = torch.empty((npq, npq), dtype=torch.float64, pin_memory=pin)
    host.copy_(e)
    del e
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    eri = host.numpy().reshape(nmo, nmo, nmo, nmo)
    vxc = rng.normal(0.0, 0.01, (nmo, nmo))
    vxc = np.triu(vxc, 1)
    vxc = vxc + vxc.T
    vxc[idx, idx] = rng.uniform(-0.6, -0.2, nmo)
    inp = GwInput(eri_mo=eri, mo_energy=mo, vxc_mo=vxc, nocc=nocc, fermi_energy=float(fermi))
    inp._pinned_owner = host  # keep the pinned tensor alive with the array view
    return inp


def make_slices_on_device(nmo: int, nocc: int, states, seed: int = 0, device: int = 0):
    """The slices of the system make_input(nmo, nocc, seed) describes (GwSlices: V_ph, the states'
    panel rows, the exchange diagonal, the vxc diagonal), computed from the Cholesky-like factors L
    with torch on the GPU, without ever forming the nmo^4 ERI (34 GB at nmo = 256).  Same random
    draws and recipe as make_input; the values differ from slices of make_input's ERI only by the
    rounding of the sums over K (V_ph is symmetrised the same way, 0.5 (A + A^T))."""
    import torch

    from .gw_input import GwSlices

    rng = np.random.default_rng(seed)
    nvir = nmo - nocc
    occ = np.sort(rng.uniform(-1.2, -0.3, nocc))
    vir = np.sort(rng.uniform(0.05, 3.0, nvir))
    mo = np.concatenate([occ, vir])
    fermi = 0.5 * (occ[-1] + vir[0])
    nk = 2 * nmo
    idx = np.arange(nmo)
    decay = 0.3 * np.exp(-np.abs(idx[:, None] - idx[None, :]) / 8.0)
    g = rng.standard_normal((nk, nmo, nmo))
    lfac = (np.triu(g) + np.transpose(np.triu(g, 1), (0, 2, 1))) * decay
    vxc = rng.normal(0.0, 0.01, (nmo, nmo))
    vxc = np.triu(vxc, 1)
    vxc = vxc + vxc.T
    vxc[idx, idx] = rng.uniform(-0.6, -0.2, nmo)
    st = np.ascontiguousarray(states, dtype=np.int64)
    n = nocc * nvir
    dev = torch.device("cuda", device)
    lt = torch.from_numpy(np.ascontiguousarray(lfac)).to(dev)          # [K, p, q]
    lov = lt[:, :nocc, nocc:].reshape(nk, n)                           # [K, ia]
    v = lov.t() @ lov
    v = 0.5 * (v + v.t())
    panel = torch.cat([lt[:, int(p), :].t() @ lov for p in st], dim=0)  # [(t, k), ia]
    xdiag = (lt[:, :, :nocc] ** 2).sum(dim=0)                          # [p, i]
    out = GwSlices(mo_energy=mo, nocc=nocc, fermi_energy=float(fermi), states=st,
                   vph=v.cpu().numpy(), panel=panel.cpu().numpy(), xdiag=xdiag.cpu().numpy(),
                   vxc_diag=np.ascontiguousarray(np.diag(vxc)))
    del lt, lov, v, panel, xdiag
    torch.cuda.empty_cache()
    return out
