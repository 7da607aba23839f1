"""gp_deposit_charge_noalloc: the allocation-free charge deposit against the
handle API's deterministic deposit of the same species (bit-identical), two
calls in a row on caller-owned device memory, with flagged records and
particles on the far walls, plus its capacity check."""
import ctypes

import numpy as np
import pytest

from gample_b200 import capi
from oracle import config as ocfg
from oracle import lib as L
from tests.helpers import condition

GP_ERR_CAPACITY = 4


def _call(order, ngx, ngy, dev_particles, n, scale, dev_rho):
    return capi.lib().gp_deposit_charge_noalloc(order, ngx, ngy, dev_particles, n, scale, dev_rho, None)


def test_noalloc_rejects_grids_beyond_its_scratch():
    # 1100 x 1100 at order 1 needs 1101^2 > 2^20 nodes: refused before any device work
    st = _call(1, 1100, 1100, None, 0, 1.0, ctypes.c_void_p(16).value)
    assert st == GP_ERR_CAPACITY
    assert b"allocation-free" in capi.lib().gp_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 3, 5])
def test_noalloc_deposit_matches_handle_api_twice_in_a_row(gpu, order):
    import torch

    ngx, ngy = 40, 28
    cond = condition(ngx=ngx, ngy=ngy, order=order, ppc=10, xbc="Dirichlet", ybc="periodic", deposit_mode=1,
                     vxe=2e7)
    sim = capi.Sim(cond)
    ora = L.OracleSim(ocfg.parse(cond))
    ngb = order // 2
    nodes = (ngx + 2 * ngb + 1) * (ngy + 2 * ngb + 1)
    rho_dev = torch.full((nodes,), float("nan"), dtype=torch.float32, device="cuda")
    # two calls in a row (electrons, then ions) on the same scratch, each
    # against the handle API's deposit of that species alone
    for s in (0, 1):
        recs = sim.particles(s)
        if s == 0:
            # flagged records (a wall code, and a negative code that is no
            # valid state) are skipped by both paths
            recs["piflag"][::97] = 1
            recs["piflag"][50::113] = -2
            # particles exactly on the far walls: the stencil nodes beyond the
            # arrays carry weight zero and are skipped
            live = np.nonzero(recs["piflag"] == 0)[0]
            recs["x"][live[3]] = np.float32(ngx + ngb)
            recs["y"][live[7]] = np.float32(ngy + ngb)
            sim.set_particles(s, recs)
        dev = torch.from_numpy(recs.view(np.uint8).copy()).cuda()
        scale = float(np.float32(ora.species_consts(s)["scale"]))
        torch.cuda.synchronize()
        assert _call(order, ngx, ngy, dev.data_ptr(), len(recs), scale, rho_dev.data_ptr()) == capi.GP_OK
        torch.cuda.synchronize()
        got = rho_dev.cpu().numpy().reshape(ngy + 2 * ngb + 1, ngx + 2 * ngb + 1)
        sim.reset_charge()
        sim.integrate_charge(s)
        want = sim.field("rho")
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), s
        assert np.count_nonzero(got) > 0
    sim.close()
