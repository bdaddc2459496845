"""Seeded synthetic workloads (no datasets are involved).

A counter-based generator (SplitMix64, Steele, Lea & Flood 2014) makes every
seeded choice, so the tests, the bench and any other caller draw identical
backgrounds and initial data from a seed.

Workloads (sizes as named in the benchmark configuration):
  * flat SIPG standing wave: unit cube, 4^3 elements, n = 6, u = sin(pi x)
    sin(pi y) sin(pi z), u_t = 0, tau = 20, KO eps = 0.1, RK4 CFL 0.25;
  * warped ADM pulse: warped cube (A = 0.05), 16^3 elements, n = 8, perturbed
    ADM background, one Gaussian pulse, Sommerfeld outer faces, RK4 CFL 0.2;
  * large warped ADM: as above at 64^3 elements (134,217,728 nodes) with eight
    Gaussian pulses (amplitude U(0.5,1), width U(0.05,0.15));
  * batched solves (batch_specs): cubic warped meshes with e ~ U{4..24}
    elements per axis and n ~ {4, 6, 8}, flat or perturbed ADM backgrounds
    with metric-perturbation amplitude U(0, 0.15), seeded pulses;
  * served solves (serve_requests): Poisson arrivals, e log-uniform in
    [4, 32], n ~ {6, 8}, final time U(0.5, 2) light-crossing times as a step
    count clamped to 200..2000 RK4 steps.
"""
from __future__ import annotations

import math

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self, a: float = 0.0, b: float = 1.0) -> float:
        return a + (b - a) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))


def adm_params(seed: int, scale: float = 1.0):
    """Parameters of the perturbed ADM background (kind BG_ADM_PERTURBED):
    alpha = 1 + 0.05 s sin(2 pi x), beta^i = 0.02 s cos(2 pi x_i),
    gamma_ij = d_ij + 0.1 s exp(-|x-c|^2/0.05)(d_ij + 0.5 s_ij), c = cube centre,
    s_ij a seeded symmetric matrix with entries U[-0.2, 0.2]; s = scale."""
    r = SplitMix64(seed)
    s = [r.uniform(-0.2, 0.2) for _ in range(6)]  # s11 s12 s13 s22 s23 s33
    return [0.05 * scale, 0.02 * scale, 0.1 * scale, 0.05, 0.5, 0.5, 0.5] + s


def _bg_eval(params, x, y, z):
    p = params
    tp = 2 * math.pi
    al = 1.0 + p[0] * np.sin(tp * x)
    b = [p[1] * np.cos(tp * x), p[1] * np.cos(tp * y), p[1] * np.cos(tp * z)]
    g = p[2] * np.exp(-((x - p[4]) ** 2 + (y - p[5]) ** 2 + (z - p[6]) ** 2) / p[3])
    s11, s12, s13, s22, s23, s33 = p[7:13]
    G = np.empty(x.shape + (3, 3))
    G[..., 0, 0] = 1 + g * (1 + 0.5 * s11); G[..., 1, 1] = 1 + g * (1 + 0.5 * s22); G[..., 2, 2] = 1 + g * (1 + 0.5 * s33)
    G[..., 0, 1] = G[..., 1, 0] = g * 0.5 * s12
    G[..., 0, 2] = G[..., 2, 0] = g * 0.5 * s13
    G[..., 1, 2] = G[..., 2, 1] = g * 0.5 * s23
    return al, b, G


def max_speed(params, npts: int = 48) -> float:
    """Bound on the coordinate characteristic speed of the perturbed ADM
    background, max(|b1| + |b2| + |b3| + sqrt(3) alpha sqrt(lambda_max(gamma^-1)))
    over a uniform npts^3 sample of the unit cube (the shape of the bound
    _background3d returns, src/evolve.jl:1119-1124)."""
    t = (np.arange(npts) + 0.5) / npts
    x, y, z = np.meshgrid(t, t, t, indexing="ij")
    al, b, G = _bg_eval(params, x, y, z)
    lam_min = np.linalg.eigvalsh(G)[..., 0]
    sp = np.abs(b[0]) + np.abs(b[1]) + np.abs(b[2]) + math.sqrt(3.0) * al / np.sqrt(lam_min)
    return float(sp.max())


def pulses(seed: int, count: int, amp=(1.0, 1.0), width=(0.1, 0.1), centre=(0.3, 0.7)):
    """count seeded Gaussian pulses: (centres (count,3), amplitudes, widths)."""
    r = SplitMix64(seed ^ 0x5DEECE66D)
    c = np.array([[r.uniform(*centre) for _ in range(3)] for _ in range(count)])
    a = np.array([r.uniform(*amp) for _ in range(count)])
    w = np.array([r.uniform(*width) for _ in range(count)])
    return c, a, w


def gaussian_field(x, y, z, centres, amps, widths):
    """Phi = sum_k A_k exp(-|x - c_k|^2 / (2 w_k^2)) (the :gaussian IC, src/evolve.jl:1260-1263)."""
    out = np.zeros_like(x)
    for c, a, w in zip(centres, amps, widths):
        out += a * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * w * w))
    return out


def gaussian_field_torch(coords, centres, amps, widths):
    """Same as gaussian_field on a device coordinate tensor of shape (nn, 3)."""
    import torch
    out = torch.zeros(coords.shape[0], dtype=torch.float64, device=coords.device)
    for c, a, w in zip(centres, amps, widths):
        d2 = ((coords - torch.tensor(c, dtype=torch.float64, device=coords.device)) ** 2).sum(dim=1)
        out += float(a) * torch.exp(-d2 / (2 * float(w) * float(w)))
    return out


def standing_wave(x, y, z):
    """u = sin(pi x) sin(pi y) sin(pi z) (eigenmode_cartesian!, src/wave.jl:163-185, k = pi)."""
    return np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)


def batch_specs(seed: int, count: int = 256, e_range=(4, 24), orders=(4, 6, 8)):
    """The batched-solve workload: count dicts with elements per axis e ~ U{e_range},
    order n ~ U(orders), background 'flat' or 'adm' (even odds) and, for 'adm',
    the metric-perturbation amplitude U(0, 0.15) (adm_params scale = amp / 0.1),
    and a pulse seed."""
    r = SplitMix64(seed ^ 0xB47C4)
    out = []
    for k in range(count):
        e = e_range[0] + min(int(r.uniform() * (e_range[1] - e_range[0] + 1)), e_range[1] - e_range[0])
        n = orders[min(int(r.uniform() * len(orders)), len(orders) - 1)]
        adm = r.uniform() < 0.5
        amp = r.uniform(0.0, 0.15) if adm else 0.0
        out.append({"elements": e, "n": n, "scale": amp / 0.1, "seed": seed * 1000 + k})
    return out


def gll_min_gap(n: int) -> float:
    """Smallest gap between the n Gauss-Lobatto-Legendre nodes on [0, 1]
    (the end nodes and the roots of P'_{n-1})."""
    inner = np.polynomial.legendre.Legendre.basis(n - 1).deriv().roots()
    x = np.sort(np.concatenate([[-1.0], inner.real, [1.0]]))
    return float(np.min(np.diff(x)) / 2.0)


def serve_requests(seed: int, count: int, rate: float, e_range=(4, 32), orders=(6, 8), steps=(200, 2000),
                   final_time=(0.5, 2.0)):
    """Served-solve requests: Poisson arrivals at `rate` per second (exponential
    gaps), e log-uniform in e_range, n ~ U(orders), ADM scale U(0, 1.5), a final
    time t ~ U(final_time) light-crossing times of the unit cube and its RK4 step
    count t / dt at CFL 0.2 (dt from the unwarped node spacing h * gll_min_gap(n)
    and the background's speed bound), clamped to the step range; and seeds for
    background and pulses."""
    r = SplitMix64(seed ^ 0x5E7E)
    t = 0.0
    out = []
    lo, hi = math.log(e_range[0]), math.log(e_range[1])
    for k in range(count):
        t += -math.log(1.0 - r.uniform()) / rate
        e = int(round(math.exp(lo + (hi - lo) * r.uniform())))
        n = orders[min(int(r.uniform() * len(orders)), len(orders) - 1)]
        tf = r.uniform(*final_time)
        scale = r.uniform(0.0, 1.5)
        rseed = seed * 100000 + k
        dt = 0.2 * gll_min_gap(n) / e / max_speed(adm_params(rseed, scale), 24)
        st = int(min(max(round(tf / dt), steps[0]), steps[1]))
        out.append({"rid": k, "arrival": t, "elements": e, "n": n, "scale": scale, "steps": st,
                    "final_time": tf, "seed": rseed})
    return out
