"""Shared builders for the tests: descriptors for small slit requests."""
from __future__ import annotations

import copy

import numpy as np

from softdft_b200 import workloads
from softdft_b200.api import setup_request


def small_slit(np_=128, dz=0.05, n_chain=6, pH=7.0, salt=0.1, eta=0.3, models=None, walls=True,
               wall_charge=None, **kw):
    ds = workloads.weak_acid_slit(np_, dz, n_chain, 4.5, pH, salt, eta, wall_charge=wall_charge, **kw)
    if models is not None:
        ds["model"] = list(models)
    if not walls:
        ds["geometry"]["external_field"] = {}
    return ds


def descriptor(ds):
    return setup_request(copy.deepcopy(ds))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def split(dft, x):
    return dft.split(x)
