"""Seeded synthetic inputs for the two hot paths.

Two families:

* the reference's own test generators, restated so the same inputs can be
  built at any size: ``a[x] = sin(x)``, ``b[x] = cos(x)`` over the flat index
  (src/impl_matmul.rs:305-306, tests/naive_matmul.rs:42-46); the AO-DM-AO test
  inputs ao_lhs = sin, ao_rhs = cos, dm = sin(0.38 x + 1.2) and the periodic
  25 % non0tab pattern with masked phi zeroed (src/impl_aodmao2rho.rs:264-296);
  the 30 % pattern of the masked GEMM test (src/impl_matmul_non0tab.rs:336-357).
* the benchmark workloads: a small Bernoulli-masked contraction (512 AOs in
  64 shells of 8, 4096 points in blocks of 64, 1 DM), the 3527x6581x9583 DGEMM,
  and a taxol-sized geometric contraction (2228 AOs in 400 s/p/d/f shells on
  110 centres, 16384 points in blocks of 64, 3 DMs, tile density 0.3).  The
  reference's README quotes its AO-DM-AO number on taxol/def2-TZVP
  (README.md:51); that basis and grid are not available here, so the
  geometric generator stands in for them with the same sizes and density.

Everything is numpy float64 / uint8, C-contiguous, and deterministic in the seed.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


# ---------------------------------------------------------------------------
# the reference tests' generators
# ---------------------------------------------------------------------------
def ref_matmul_inputs(m: int, n: int, k: int, transa: bool = False, transb: bool = False):
    """A[x] = sin(x), B[x] = cos(x) on the flat index with ld = row length,
    as in test_matmul_anyway_full / _transb / _transa (impl_matmul.rs:297-397)."""
    a_rows, a_cols = (k, m) if transa else (m, k)
    b_rows, b_cols = (n, k) if transb else (k, n)
    a = np.sin(np.arange(a_rows * a_cols, dtype=np.float64)).reshape(a_rows, a_cols)
    b = np.cos(np.arange(b_rows * b_cols, dtype=np.float64)).reshape(b_rows, b_cols)
    return a, b, a_cols, b_cols  # lda, ldb


MOD_PATTERN_25 = np.array([1, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 0, 0, 1, 0], np.uint8)
MOD_PATTERN_30 = np.array([1, 0, 1, 0, 0, 1, 0, 0, 0, 0], np.uint8)


def ref_aodmao2rho_inputs(nao: int, ngrid: int, nset: int = 1, blksize: int = 48,
                          dense: bool = False):
    """Inputs of test_aodmao2rho_1 / test_aodmao2rho_all_dense
    (impl_aodmao2rho.rs:264-296, 348-380) at any size: ao_lhs = sin, ao_rhs =
    cos, dm = sin(0.38 x + 1.2) (not symmetric), the 25 % periodic non0tab
    (or all true), and phi zeroed in masked (AO, block) tiles."""
    nblk = -(-ngrid // blksize)
    x = np.arange(nao * ngrid, dtype=np.float64)
    ao_lhs = np.sin(x).reshape(nao, ngrid)
    ao_rhs = np.cos(x).reshape(nao, ngrid)
    dm = np.sin(np.arange(nset * nao * nao, dtype=np.float64) * 0.38 + 1.2).reshape(nset, nao, nao)
    if dense:
        tab = np.ones((nao, nblk), np.uint8)
    else:
        tab = MOD_PATTERN_25[np.arange(nao * nblk) % 20].reshape(nao, nblk).copy()
    mask = expand_mask(tab, ngrid, blksize)
    ao_lhs[~mask] = 0.0
    ao_rhs[~mask] = 0.0
    return ao_lhs, ao_rhs, dm, tab, nblk


def ref_matmul_non0tab_inputs(m: int, n: int, k: int, blksize: int = 48):
    """Inputs of test_matmul_anyway_full_non0tab (impl_matmul_non0tab.rs:328-357)."""
    a, b, lda, ldb = ref_matmul_inputs(m, n, k)
    nblk = -(-n // blksize)
    tab = MOD_PATTERN_30[np.arange(k * nblk) % 10].reshape(k, nblk).copy()
    b[~expand_mask(tab, n, blksize)] = 0.0
    return a, b, lda, ldb, tab, nblk


def expand_mask(tab: np.ndarray, ngrid: int, blksize: int) -> np.ndarray:
    """(nao, nblk) block mask -> (nao, ngrid) bool point mask."""
    return np.repeat(tab.astype(bool), blksize, axis=1)[:, :ngrid]


def dense_rho(ao_lhs, ao_rhs, dms, tab, blksize):
    """rho by dense FP64 linear algebra on masked phi: the comparator of the
    reference's tests (dm @ ao_rhs, times ao_lhs, summed over AOs;
    impl_aodmao2rho.rs:303-345)."""
    nao, ngrid = ao_lhs.shape
    mask = expand_mask(tab, ngrid, blksize)
    L = np.where(mask, ao_lhs, 0.0)
    R = np.where(mask, ao_rhs, 0.0)
    return np.stack([(L * (d @ R)).sum(axis=0) for d in dms])


def masked_flops(tab: np.ndarray, ngrid: int, blksize: int, nset: int) -> float:
    """Algorithmic FLOPs of the masked contraction:
    sum_s sum_b (2 |I_b|^2 + 2 |I_b|) * |b| (a GEMM of |I_b| x |I_b| x |b|
    plus the fused multiply-reduce over u)."""
    nb = tab.astype(bool).sum(axis=0).astype(np.float64)
    nblk = tab.shape[1]
    sizes = np.full(nblk, float(blksize))
    sizes[-1] = ngrid - blksize * (nblk - 1)
    return float(nset * np.sum((2.0 * nb * nb + 2.0 * nb) * sizes))


def symmetric_flops(tab: np.ndarray, ngrid: int, blksize: int, nset: int,
                    tile: int = 64) -> float:
    """FLOPs the FP64 kernel's symmetric-D mode executes: row tile a of a block
    (|I_b| compacted AOs in tiles of `tile`) contracts the compacted columns from
    a*tile on, sum_s sum_b |b| (sum_a 2 m_a (|I_b| - a*tile) + 2 |I_b|) with
    m_a = min(tile, |I_b| - a*tile)."""
    nb = tab.astype(bool).sum(axis=0).astype(np.int64)
    nblk = tab.shape[1]
    sizes = np.full(nblk, float(blksize))
    sizes[-1] = ngrid - blksize * (nblk - 1)
    tot = 0.0
    for n, w in zip(nb, sizes):
        k = 0.0
        for a0 in range(0, int(n), tile):
            k += 2.0 * min(tile, n - a0) * (n - a0)
        tot += (k + 2.0 * n) * w
    return float(nset * tot)


# ---------------------------------------------------------------------------
# benchmark workloads
# ---------------------------------------------------------------------------
@dataclass
class AodmProblem:
    ao: np.ndarray      # (nao, ngrid) float64; ao_lhs = ao_rhs = ao
    dms: np.ndarray     # (nset, nao, nao) float64, symmetric
    tab: np.ndarray     # (nao, nblk) uint8
    blksize: int
    shell_sizes: np.ndarray
    name: str

    @property
    def nao(self): return self.ao.shape[0]

    @property
    def ngrid(self): return self.ao.shape[1]

    @property
    def nset(self): return self.dms.shape[0]

    @property
    def nblk(self): return self.tab.shape[1]

    def flops(self) -> float:
        return masked_flops(self.tab, self.ngrid, self.blksize, self.nset)

    def density(self) -> float:
        return float(self.tab.mean())


def sym_dms(rng, nset: int, nao: int) -> np.ndarray:
    a = rng.uniform(-1.0, 1.0, (nset, nao, nao))
    return np.ascontiguousarray(0.5 * (a + a.transpose(0, 2, 1)))


def small_masked(seed: int = 0, nao: int = 512, shell: int = 8, ngrid: int = 4096,
                 blksize: int = 64, nset: int = 1, density: float = 0.3) -> AodmProblem:
    """nao AOs in shells of `shell`, ngrid points in blocks of `blksize`; the
    (shell, block) mask is Bernoulli(density); phi ~ N(0,1) inside unmasked
    tiles and exactly 0 elsewhere; D = (A + A^T)/2, A ~ U(-1, 1)."""
    rng = np.random.default_rng(seed)
    nsh = nao // shell
    nblk = -(-ngrid // blksize)
    sh_tab = (rng.random((nsh, nblk)) < density).astype(np.uint8)
    tab = np.repeat(sh_tab, shell, axis=0)
    ao = rng.standard_normal((nao, ngrid))
    ao[~expand_mask(tab, ngrid, blksize)] = 0.0
    return AodmProblem(ao, sym_dms(rng, nset, nao), np.ascontiguousarray(tab), blksize,
                       np.full(nsh, shell), f"bernoulli nao={nao} ngrid={ngrid} nset={nset}")


def _solid_harmonics(l: int, x, y, z):
    """Real solid harmonics r^l Y_lm (unnormalised polynomials) for l = 0..3."""
    if l == 0:
        return [np.ones_like(x)]
    if l == 1:
        return [x, y, z]
    r2 = x * x + y * y + z * z
    if l == 2:
        return [x * y, y * z, 3 * z * z - r2, x * z, x * x - y * y]
    return [y * (3 * x * x - y * y), x * y * z, y * (5 * z * z - r2), z * (5 * z * z - 3 * r2),
            x * (5 * z * z - r2), z * (x * x - y * y), x * (x * x - 3 * y * y)]


def shell_sizes_for(rng, nshell: int, nao: int) -> np.ndarray:
    """Shell sizes drawn from {1,3,5,7} (s,p,d,f) with weights that favour the
    target mean, then fixed up by +-2 steps until they sum to exactly nao."""
    sizes = rng.choice([1, 3, 5, 7], size=nshell, p=[0.05, 0.15, 0.3, 0.5])
    diff = nao - int(sizes.sum())
    if diff % 2:
        raise ValueError("nao must have the parity of nshell for odd shell sizes")
    while diff != 0:
        i = int(rng.integers(nshell))
        if diff > 0 and sizes[i] < 7:
            sizes[i] += 2
            diff -= 2
        elif diff < 0 and sizes[i] > 1:
            sizes[i] -= 2
            diff += 2
    return sizes


@dataclass
class Molecule:
    """Shells of Gaussian AOs on atom centres (AOs ordered by centre)."""
    centres: np.ndarray      # (natom, 3) bohr
    shell_atom: np.ndarray   # (nshell,)
    shell_l: np.ndarray      # (nshell,) angular momentum 0..3
    alpha: np.ndarray        # (nshell,) bohr^-2
    sizes: np.ndarray        # (nshell,) 2l+1

    @property
    def nao(self): return int(self.sizes.sum())

    @property
    def nshell(self): return len(self.sizes)

    @property
    def rows(self): return np.concatenate([[0], np.cumsum(self.sizes)[:-1]]).astype(np.int32)

    @property
    def norm(self):
        a, l = self.alpha, self.shell_l
        return (2 * a / np.pi) ** 0.75 * (4 * a) ** (l / 2)

    @property
    def shell_xyz(self): return np.ascontiguousarray(self.centres[self.shell_atom])


def molecule(seed: int = 0, nao: int = 2228, nshell: int = 400, natom: int = 110,
             box_angstrom: float = 16.0) -> Molecule:
    """natom centres uniform in a cube of `box_angstrom`; shells of sizes
    1,3,5,7 (s,p,d,f) summing to nao, sorted onto centres; exponents
    log-uniform in [0.05, 20] bohr^-2."""
    rng = np.random.default_rng(seed)
    box = box_angstrom / 0.529177210903
    centres = rng.uniform(0.0, box, (natom, 3))
    sizes = shell_sizes_for(rng, nshell, nao)
    shell_atom = np.sort(rng.integers(0, natom, nshell))
    alpha = np.exp(rng.uniform(np.log(0.05), np.log(20.0), nshell))
    return Molecule(centres, shell_atom, (sizes - 1) // 2, alpha, sizes)


def grid_points(rng, mol: Molecule, ngrid: int, blksize: int) -> np.ndarray:
    """Each block of `blksize` points is sampled around one centre (Gaussian
    offsets, sigma 1.5 bohr), as atom-centred DFT grids grouped into blocks are."""
    nblk = -(-ngrid // blksize)
    blk_atom = rng.integers(0, len(mol.centres), nblk)
    return mol.centres[np.repeat(blk_atom, blksize)[:ngrid]] + rng.normal(0.0, 1.5, (ngrid, 3))


def eval_ao_numpy(mol: Molecule, pts: np.ndarray) -> np.ndarray:
    """phi[row + f][g] = N exp(-alpha r^2) Y_f, Y_f the real solid harmonics."""
    ao = np.empty((mol.nao, len(pts)))
    rows, norm = mol.rows, mol.norm
    for s in range(mol.nshell):
        d = pts - mol.centres[mol.shell_atom[s]]
        x, y, z = d[:, 0], d[:, 1], d[:, 2]
        radial = norm[s] * np.exp(-mol.alpha[s] * (x * x + y * y + z * z))
        for f, h in enumerate(_solid_harmonics(int(mol.shell_l[s]), x, y, z)):
            ao[rows[s] + f] = radial * h
    return ao


def shell_block_max(mol: Molecule, ao: np.ndarray, blksize: int) -> np.ndarray:
    nao, ngrid = ao.shape
    nblk = -(-ngrid // blksize)
    absao = np.abs(ao)
    pad = nblk * blksize - ngrid
    if pad:
        absao = np.concatenate([absao, np.zeros((nao, pad))], axis=1)
    blkmax = absao.reshape(nao, nblk, blksize).max(axis=2)
    return np.maximum.reduceat(blkmax, mol.rows, axis=0)


def density_threshold(shmax: np.ndarray, density: float) -> float:
    """Threshold keeping the `density` fraction of (shell, block) tiles."""
    return float(np.quantile(shmax, 1.0 - density))


def geometric(seed: int = 0, nao: int = 2228, nshell: int = 400, natom: int = 110,
              ngrid: int = 16384, blksize: int = 64, nset: int = 3, density: float = 0.3,
              box_angstrom: float = 16.0) -> AodmProblem:
    """Taxol-sized geometric contraction (numpy): molecule(seed) and a grid
    drawn from the same seed; the (shell, block) mask keeps the `density`
    fraction of tiles with the largest max|phi|; phi is zeroed elsewhere."""
    mol = molecule(seed, nao, nshell, natom, box_angstrom)
    rng = np.random.default_rng(seed + 1_000_003)
    pts = grid_points(rng, mol, ngrid, blksize)
    ao = eval_ao_numpy(mol, pts)
    shmax = shell_block_max(mol, ao, blksize)
    sh_tab = (shmax > density_threshold(shmax, density)).astype(np.uint8)
    tab = np.repeat(sh_tab, mol.sizes, axis=0)
    ao[~expand_mask(tab, ngrid, blksize)] = 0.0
    return AodmProblem(np.ascontiguousarray(ao), sym_dms(rng, nset, nao),
                       np.ascontiguousarray(tab), blksize, mol.sizes,
                       f"geometric nao={nao} ngrid={ngrid} nset={nset}")


# ---------------------------------------------------------------------------
# device-side generation through the library's AO evaluator
# ---------------------------------------------------------------------------
class DeviceMolecule:
    """A Molecule's shell arrays on the device, for cfgmm_eval_ao_dev."""

    def __init__(self, mol: Molecule, device="cuda"):
        import torch
        self.mol = mol
        self.xyz = torch.from_numpy(mol.shell_xyz).to(device)
        self.l = torch.from_numpy(mol.shell_l.astype(np.int32)).to(device)
        self.alpha = torch.from_numpy(mol.alpha.astype(np.float64)).to(device)
        self.norm = torch.from_numpy(mol.norm.astype(np.float64)).to(device)
        self.row = torch.from_numpy(mol.rows).to(device)


def device_grid(cm, dmol: DeviceMolecule, pts: np.ndarray, blksize: int, density: float):
    """phi (nao, ngrid) and tab (nao, nblk) on the device: AOs evaluated by the
    library, mask at the `density` quantile of the (shell, block) maxima."""
    import torch
    mol = dmol.mol
    ngrid = len(pts)
    nblk = -(-ngrid // blksize)
    dev = dmol.xyz.device
    p = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
    ao = torch.empty(mol.nao, ngrid, dtype=torch.float64, device=dev)
    bmax = torch.empty(mol.nshell, nblk, dtype=torch.float64, device=dev)
    tab = torch.empty(mol.nao, nblk, dtype=torch.uint8, device=dev)
    cm.eval_ao(ao, p, dmol.xyz, dmol.l, dmol.alpha, dmol.norm, dmol.row, bmax, blksize)
    thr = float(torch.quantile(bmax.flatten(), 1.0 - density))
    cm.mask_ao(ao, ngrid, dmol.l, dmol.row, bmax, thr, tab, blksize)
    return ao, tab


@dataclass
class BatchedProblem:
    mol: Molecule
    dms: object             # torch (nset_max, nao, nao)
    batches: list           # [(ao, tab, ngrid, nset, density)] device tensors
    blksize: int

    def flops(self) -> float:
        tot = 0.0
        for ao, tab, ngrid, nset, _ in self.batches:
            tot += masked_flops(tab.cpu().numpy(), ngrid, self.blksize, nset)
        return tot

    def points(self) -> int:
        return sum(b[2] for b in self.batches)


def batched_uneven(cm, seed: int = 0, nbatch: int = 256, nao: int = 2228, nshell: int = 400,
                   natom: int = 110, gmin: int = 128, gmax: int = 4096, dmin: float = 0.05,
                   dmax: float = 0.6, nset_max: int = 3, blksize: int = 64) -> BatchedProblem:
    """Uneven grid batches of one taxol-sized molecule: ngrid log-uniform in
    [gmin, gmax], tile density uniform in [dmin, dmax], 1..nset_max DMs each;
    phi and masks evaluated on the device."""
    import torch
    mol = molecule(seed, nao, nshell, natom)
    rng = np.random.default_rng(seed + 7)
    dmol = DeviceMolecule(mol)
    batches = []
    for _ in range(nbatch):
        ngrid = int(np.exp(rng.uniform(np.log(gmin), np.log(gmax))))
        dens = float(rng.uniform(dmin, dmax))
        nset = int(rng.integers(1, nset_max + 1))
        ao, tab = device_grid(cm, dmol, grid_points(rng, mol, ngrid, blksize), blksize, dens)
        batches.append((ao, tab, ngrid, nset, dens))
    dms = torch.from_numpy(sym_dms(rng, nset_max, nao)).cuda()
    return BatchedProblem(mol, dms, batches, blksize)


def dgemm_uniform(m: int = 3527, n: int = 9583, k: int = 6581, transa: bool = False,
                  transb: bool = False, seed: int = 0):
    """A, B ~ U(-1, 1) with ld = row length (op(A) is m x k, op(B) is k x n)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1.0, 1.0, (k, m) if transa else (m, k))
    b = rng.uniform(-1.0, 1.0, (n, k) if transb else (k, n))
    return a, b, a.shape[1], b.shape[1]
