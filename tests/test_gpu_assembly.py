"""Bond-parameter assembly upstream of the 3D solve (train3d.Scatter, train3d.group_penalty on the CUDA library)
against the reference's own outputs and autograd gradients (tests/golden/golden_asm.npz, made by running
coarse3d/train3d.py on the CPU).  Bars: scatter bit-exact, penalty and gradients 1e-10 relative."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, relmax
from lpm_b200 import torch_lpm3d as T3
from lpm_b200 import train3d as TR

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


@pytest.fixture(scope="module")
def ga():
    with np.load(os.path.join(GOLDEN, "golden_asm.npz")) as d:
        return {k: d[k] for k in d.files}


def leaves(ga):
    out = []
    for i in range(2):
        out += [torch.tensor(ga["kn%d" % i], device=DEV, requires_grad=True),
                torch.tensor(ga["tv%d" % i], device=DEV, requires_grad=True)]
    return out


def test_bond_groups_match_reference(ga):
    cm = T3.CoarseT(5, 2, device=DEV)
    groups = TR.forward_bond_groups(cm.lat)
    for i in range(2):
        assert np.array_equal(groups[i]["bonds"], ga["bonds%d" % i])


def test_scatter_and_its_gradient(ga):
    groups = [dict(bonds=ga["bonds%d" % i]) for i in range(2)]
    sc = TR.Scatter(5, 2, groups, device=DEV)
    lv = leaves(ga)
    Kn, Tv = sc([(lv[0], lv[1]), (lv[2], lv[3])])
    assert np.array_equal(Kn.detach().cpu().numpy(), ga["Kn"]) and np.array_equal(Tv.detach().cpu().numpy(), ga["Tv"])
    Ls = (Kn * torch.tensor(ga["Wk"], device=DEV)).sum() + (Tv * torch.tensor(ga["Wt"], device=DEV)).sum()
    gs = torch.autograd.grad(Ls, lv)
    for i in range(2):
        assert relmax(gs[2 * i].cpu().numpy(), ga["gs_kn%d" % i]) < 1e-14
        assert relmax(gs[2 * i + 1].cpu().numpy(), ga["gs_tv%d" % i]) < 1e-14


def test_group_penalty_and_its_gradient(ga):
    cm = T3.CoarseT(5, 2, device=DEV)
    groups = [dict(bonds=ga["bonds%d" % i]) for i in range(2)]
    sc = TR.Scatter(5, 2, groups, device=DEV)
    lv = leaves(ga)
    Kn, Tv = sc([(lv[0], lv[1]), (lv[2], lv[3])])
    pen, lmin = TR.group_penalty(cm, Kn, Tv, frac=0.05)
    assert relmax(pen.detach().cpu().numpy(), ga["pen"]) < 1e-10
    assert abs(lmin - float(ga["lmin"])) < 1e-10 * abs(float(ga["lmin"]))
    gp = torch.autograd.grad(pen.sum(), lv)
    for i in range(2):
        assert relmax(gp[2 * i].cpu().numpy(), ga["gp_kn%d" % i]) < 1e-8
        assert relmax(gp[2 * i + 1].cpu().numpy(), ga["gp_tv%d" % i]) < 1e-8
