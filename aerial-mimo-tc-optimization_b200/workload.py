"""Seeded synthetic PUSCH slots for the equalization path.

No public dataset is involved: the workloads are the shapes and channel /
noise models of the five benchmark configurations, generated from a seed
with torch's generator (on CPU for the parity tests, on the GPU for large
benchmark batches; the two streams differ, each run is self-consistent).

Conventions:
  - Tx symbols: Gray-mapped square QAM with 2*nPamBits bits per symbol, unit
    average energy, per real dimension sb_{n-1} = (1-2b_{n-1}) D_{n-1},
    sb_i = (1-2b_i)(D_i - sb_{i+1}); this is the mapping the max-log demapper
    of src/llr/aerial_llr_v3.cu:84-108 inverts (bit i = 1 <-> sb_i < 0).
  - H[sc][ant][layer] with E|h|^2 = 1/nAnt, so each layer arrives with unit
    combined gain and SNR = 1/sigma2 is the per-layer post-combining SNR;
    sigma2 = 10^(-SNR/10) is the complex noise variance per antenna.
  - Y_rx[sc][sym][ant] = sum_l H[sc][ant][l] x[sc][l][sym] + CN(0, sigma2).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch

QAM_BITS = {4: 1, 16: 2, 64: 3, 256: 4}   # QAM order -> nPamBits


def pam_distances(n: int):
    """D_i = 2^(n-1-i) / sqrt(2(4^n-1)/3), i = 0..n-1."""
    norm = math.sqrt(2.0 * (4 ** n - 1) / 3.0)
    return [2 ** (n - 1 - i) / norm for i in range(n)]


def pam_map(bits: torch.Tensor) -> torch.Tensor:
    """bits[..., n] (0/1) -> PAM amplitude[...] (float32)."""
    n = bits.shape[-1]
    D = pam_distances(n)
    b = bits.to(torch.float32)
    sb = (1 - 2 * b[..., n - 1]) * D[n - 1]
    for i in range(n - 2, -1, -1):
        sb = (1 - 2 * b[..., i]) * (D[i] - sb)
    return sb


@dataclass
class Cell:
    """One cell-slot: inputs, truth and shape."""
    H: torch.Tensor          # complex64 [nSC, nAnt, L]
    Y: torch.Tensor          # complex64 [nSC, nSym, nAnt]
    bits: torch.Tensor       # uint8 [nSC, L, nSym, nPamBits, 2]  (bit, iq) like the LLR order
    x: torch.Tensor          # complex64 [nSC, L, nSym]
    sigma2: float
    nPRB: int
    nAnt: int
    nLayers: int
    nSym: int
    nPamBits: int
    snr_db: float

    @property
    def nSC(self) -> int:
        return 12 * self.nPRB

    @property
    def n_re(self) -> int:
        return self.nSC * self.nSym

    @property
    def llr_numel(self) -> int:
        return self.nSC * self.nLayers * self.nSym * 2 * self.nPamBits

    def algorithmic_bytes(self) -> int:
        """H + Y_rx read as complex64, LLRs written as float32."""
        return 8 * self.nSC * self.nAnt * self.nLayers + 8 * self.nSC * self.nSym * self.nAnt + 4 * self.llr_numel


def _cn(shape, var, gen, device):
    s = math.sqrt(var / 2.0)
    re = torch.randn(shape, generator=gen, device=device) * s
    im = torch.randn(shape, generator=gen, device=device) * s
    return torch.complex(re, im)


def make_cell(nPRB=132, nAnt=64, nLayers=8, nSym=11, qam=256, snr_db=25.0, channel="iid", rho=0.7,
              perturb=0.01, seed=42, device="cpu") -> Cell:
    """Generate one cell-slot.

    channel: "iid"  H ~ CN(0, 1/nAnt) per subcarrier
             "prb"  CN(0, 1/nAnt) constant over each 12-subcarrier PRB plus a
                    per-subcarrier CN(0, perturb/nAnt) perturbation
             "corr" H = R^(1/2) G, G ~ CN(0, 1/nAnt), R_ij = rho^|i-j| over antennas
    """
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    nSC = 12 * nPRB
    n = QAM_BITS[qam]
    if channel == "iid":
        H = _cn((nSC, nAnt, nLayers), 1.0 / nAnt, gen, device)
    elif channel == "prb":
        Hp = _cn((nPRB, 1, nAnt, nLayers), 1.0 / nAnt, gen, device).expand(nPRB, 12, nAnt, nLayers)
        H = (Hp.reshape(nSC, nAnt, nLayers) + _cn((nSC, nAnt, nLayers), perturb / nAnt, gen, device))
    elif channel == "corr":
        idx = torch.arange(nAnt, device=device, dtype=torch.float64)
        R = rho ** (idx[:, None] - idx[None, :]).abs()
        evals, evecs = torch.linalg.eigh(R)
        Rh = (evecs * evals.clamp_min(0).sqrt()) @ evecs.T
        G = _cn((nSC, nAnt, nLayers), 1.0 / nAnt, gen, device)
        H = torch.matmul(Rh.to(torch.complex64), G)
    else:
        raise ValueError(channel)
    H = H.to(torch.complex64).contiguous()
    bits = torch.randint(0, 2, (nSC, nLayers, nSym, n, 2), generator=gen, device=device, dtype=torch.uint8)
    xi = pam_map(bits[..., 0])
    xq = pam_map(bits[..., 1])
    x = torch.complex(xi, xq)                                   # [nSC, L, nSym]
    sigma2 = 10.0 ** (-snr_db / 10.0)
    # Y[sc][s][a] = sum_l H[sc][a][l] x[sc][l][s]
    Y = torch.matmul(H, x).transpose(1, 2)                      # [nSC, nSym, nAnt]
    Y = (Y + _cn((nSC, nSym, nAnt), sigma2, gen, device)).to(torch.complex64).contiguous()
    return Cell(H, Y, bits, x.to(torch.complex64), float(sigma2), nPRB, nAnt, nLayers, nSym, n, float(snr_db))


# ---------------------------------------------------------------------------
# benchmark configurations
# ---------------------------------------------------------------------------

def config_cell(cfg: int, seed: int = 42, device="cpu") -> Cell:
    """Configurations 1-3 (single cell)."""
    if cfg == 1:
        return make_cell(24, 32, 4, 11, 16, 20.0, "iid", seed=seed, device=device)
    if cfg == 2:
        return make_cell(132, 64, 8, 11, 256, 25.0, "prb", seed=seed, device=device)
    if cfg == 3:
        return make_cell(273, 128, 16, 11, 256, 30.0, "corr", seed=seed, device=device)
    raise ValueError(cfg)


def multicell_shapes(n_cells=16, seed=42):
    """Configuration 4: per-cell (nPRB, nAnt, nLayers, qam, snr_db) drawn from a seed."""
    g = torch.Generator()
    g.manual_seed(int(seed))
    prbs, ants, layers, qams = [24, 51, 106, 132, 273], [16, 32, 64], [2, 4, 8], [4, 16, 64, 256]
    out = []
    for _ in range(n_cells):
        p = prbs[int(torch.randint(len(prbs), (1,), generator=g))]
        a = ants[int(torch.randint(len(ants), (1,), generator=g))]
        l = layers[int(torch.randint(len(layers), (1,), generator=g))]
        q = qams[int(torch.randint(len(qams), (1,), generator=g))]
        snr = 10.0 + 20.0 * float(torch.rand((1,), generator=g))
        out.append((p, a, l, q, snr))
    return out


def multicell(n_cells=16, seed=42, device="cpu"):
    return [make_cell(p, a, l, 11, q, snr, "iid", seed=seed + 1000 * i, device=device)
            for i, (p, a, l, q, snr) in enumerate(multicell_shapes(n_cells, seed))]
