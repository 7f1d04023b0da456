"""Algorithmic HBM bytes of one Anderson iteration of one request.

One definition, used by bench.py for ``roofline.achieved``.  With P grid
points, NB bead types, MB bond types, per species u its N_u segments and S_u
states, Anderson depth m, n = P (NB + 2 MB + 1) + 1 unknowns, w_p the
propagator/convolution element size (8 in FP64, 4 in the mixed form):

    B_iter = 8 P (2 NB + 1)                                    lambda: read mu, Ext; write lambda
           + sum_u w_p P 2 (N_u - 1)(2 S_u + 2 S_u^2)           propagator steps: read lambda, previous
                                                                 propagator sums and ln g; write gC / gP
           + sum_u [ w_p P (2 N_u S_u^2 + N_u S_u)
                     + 8 P (N_u S_u + 2 MB) ]                    density assembly: read gC+gP, lambda;
                                                                 write rho_seg, rho_bonds
           + 8 P (sum_u N_u S_u + NB)                           bead densities
           + 8 P (NB + 2 MB)                                    densities read by the functionals
           + 8 P (NB + 2 MB + 1)                                write mu_ex, ln g, Psi
           + 8 n (2 m + 4)                                      Anderson: read histories, write columns,
                                                                 read/write x

FFT intermediates, weighted densities and the zero vector components of the 1D
weights are not counted (they live in shared memory or are never formed).
"""
from __future__ import annotations

from .host.descriptor import Descriptor


def algorithmic_bytes_per_iteration(d: Descriptor, anderm: int, w_p: int = 8) -> int:
    P, NB, MB = d.np_, d.nb, d.mb
    n = P * (NB + 2 * MB + 1) + 1
    b = 8 * P * (2 * NB + 1)
    for u in range(d.n_species):
        N, S = d.n_seg[u], d.max_states[u]
        b += w_p * P * 2 * (N - 1) * (2 * S + 2 * S * S)
        b += w_p * P * (2 * N * S * S + N * S) + 8 * P * (N * S + 2 * MB)
    b += 8 * P * (sum(d.n_seg[u] * d.max_states[u] for u in range(d.n_species)) + NB)
    b += 8 * P * (NB + 2 * MB)
    b += 8 * P * (NB + 2 * MB + 1)
    b += 8 * n * (2 * anderm + 4)
    return int(b)
