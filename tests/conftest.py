"""Shared pytest setup: the ``gpu`` marker, import paths and small problems."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import efie_oracle as eo  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pkg():
    return importlib.import_module("matlab-cuda-efief-vs-cpu_b200")


def small_design(order="grid", opts=None, npx=4, npy=3, ngx=6, ngy=6, h=1.6e-3):
    """A small two-plate problem (Ne ~ 125) for fast parity checks."""
    return eo.Design(Lp=12e-3, Wp=16e-3, Lg=30e-3, Wg=30e-3, h=h, Np_x=npx, Np_y=npy, Ng_x=ngx, Ng_y=ngy,
                     feed=(0.0, -2e-3), vertex_order=order,
                     opts=dict(opts or eo.DEFAULT_OPTS_GPU), freqs=np.linspace(2e9, 3e9, 3))


def config1_design(order="grid", opts=None):
    """Patch 38x30 mm as a 12x10 grid, ground 60x60 mm as 16x16, h = 1.6 mm (Ne = 1074)."""
    return eo.Design(Lp=30e-3, Wp=38e-3, Lg=60e-3, Wg=60e-3, h=1.6e-3, Np_x=12, Np_y=10, Ng_x=16, Ng_y=16,
                     feed=(0.0, -7e-3), vertex_order=order, opts=dict(opts or eo.DEFAULT_OPTS_GPU),
                     freqs=np.linspace(2e9, 3e9, 11))


@pytest.fixture(scope="session")
def small_problem():
    return eo.build_problem(small_design())


@pytest.fixture(scope="session")
def ref_problem():
    """The reference's own GPU sweep design (Ne = 538)."""
    return eo.build_problem(eo.reference_sweep_design())
