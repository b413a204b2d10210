"""Known answers of the standard-boundary specification (oracle_std_* in
oracle/imexlb_oracle.c), which the device's standard boundaries are checked
against bit for bit.  None of them needs reference code: each is a property
of the exact equations that halfway bounce-back keeps to round-off.

* A closed cavity with a moving lid conserves its mass, sum of 3p: the lid
  term 6 w_q rho_w (e_q . u_w) sums to zero over the links of each lid cell.
* A cavity whose lid is at rest stays exactly at rest.
* A sphere channel without solid cells stays at the uniform inflow
  equilibrium (inlet, outlet and periodic sides all hand it back).
* The lid-driven slab (the cavity's bottom wall and lid, x and y periodic)
  reaches plane Couette flow, u(z) = u_w (z + 1/2) / nz with the walls
  half a cell outside the first and last planes, for any relaxation time.
"""
import numpy as np
import pytest

from oracle.bindings import OracleStd


def test_moving_lid_cavity_conserves_mass():
    o = OracleStd("cavity", 20, 18, 22, 0.06, 1.0, 0.1, lid_u=0.1)
    for _ in range(4):
        o.step(100)
        u, v, w, p = o.moments()
        assert abs((3 * p).sum()) <= 1e-13 * np.abs(3 * p).sum()
        assert np.abs(u).max() > 0.05  # the lid drives the flow


def test_cavity_at_rest_stays_at_rest():
    o = OracleStd("cavity", 12, 10, 14, 0.06, 1.0, 0.0, lid_u=0.0)
    o.step(200)
    for a in o.moments():
        assert np.all(a == 0.0)


def test_channel_without_solid_stays_uniform():
    # a sphere of diameter 1e-3 centred between cells covers no cell
    o = OracleStd("sphere", 40, 12, 14, 0.05, 1.0, 0.05, inlet_u=0.05, sphere_d=1e-3, sphere_c=(10.5, 6.5, 7.5))
    o.step(300)
    u, v, w, p = o.moments()
    assert np.abs(u - 0.05).max() <= 1e-14
    assert max(np.abs(v).max(), np.abs(w).max(), np.abs(p).max()) <= 1e-14


@pytest.mark.parametrize("nz,tau0,steps", [(8, 0.5, 6000), (8, 0.2, 20000), (6, 1.5, 4000)])
def test_slab_reaches_plane_couette_flow(nz, tau0, steps):
    lid = 0.04
    o = OracleStd("slab", 4, 3, nz, tau0, 1.0, lid, lid_u=lid)
    o.step(steps)
    u, v, w, p = o.moments()
    want = lid * (np.arange(nz) + 0.5) / nz
    assert np.abs(u - want[:, None, None]).max() <= 1e-14
    assert max(np.abs(v).max(), np.abs(w).max()) <= 1e-15
