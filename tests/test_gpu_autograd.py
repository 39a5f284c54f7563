"""torch.autograd through the device einsum (the counterpart of the
reference's rrule, src/autodiff.jl:35-44): gradients of a scalar loss match
those of torch.einsum in FP64 on the host (a plain PyTorch reference of the
same operation), for flat and nested codes, real and complex inputs."""
import numpy as np
import pytest
import torch

import omeinsum_b200 as ome

pytestmark = pytest.mark.gpu

CASES = [
    ("ij,jk->ik", None),
    ("ij,jk,kl->il", None),
    ("(ij,jk),kl->il", "nested"),
    ("ijk,jkl->il", None),
    ("ii->i", None),
    ("ij,ij->", None),
]


def _torch_code(code):
    return code.replace("(", "").replace(")", "")


@pytest.mark.parametrize("dtype", [torch.float64, torch.complex128, torch.float32])
@pytest.mark.parametrize("code,kind", CASES)
def test_gradients_match_torch(code, kind, dtype):
    g = torch.Generator().manual_seed(3)
    flat = _torch_code(code)
    lhs, iy = flat.split("->")
    ixs = lhs.split(",")
    sd = {l: 3 + (ord(l) % 3) for l in set("".join(ixs))}
    xs_h = [torch.randn([sd[l] for l in ix], generator=g, dtype=torch.float64) for ix in ixs]
    if dtype.is_complex:
        xs_h = [x + 1j * torch.randn(x.shape, generator=g, dtype=torch.float64) for x in xs_h]
    w_h = torch.randn([sd[l] for l in iy], generator=g, dtype=torch.float64)
    # host reference (FP64 / complex128)
    ref_in = [x.clone().requires_grad_(True) for x in xs_h]
    yr = torch.einsum(flat, *ref_in)
    loss_r = (yr * w_h).real.sum() if yr.is_complex() else (yr * w_h).sum()
    loss_r.backward()
    # device
    dev_in = [x.to("cuda", dtype).requires_grad_(True) for x in xs_h]
    c = ome.ein(code) if kind == "nested" else ome.EinCode([tuple(ix) for ix in ixs], tuple(iy))
    y = ome.ad_einsum(c, dev_in)
    wd = w_h.to("cuda", dtype if not dtype.is_complex else torch.float64)
    loss = (y * wd).real.sum() if y.is_complex() else (y * wd).sum()
    loss.backward()
    ome.device_status()
    tol = 1e-5 if dtype == torch.float32 else 1e-10
    assert abs(loss.item() - loss_r.item()) <= tol * max(1.0, abs(loss_r.item()))
    for a, b in zip(dev_in, ref_in):
        ga, gb = a.grad.detach().cpu().to(torch.complex128 if dtype.is_complex else torch.float64), b.grad
        assert torch.linalg.norm(ga - gb) <= tol * max(torch.linalg.norm(gb).item(), 1e-300)


def test_only_requested_inputs_get_gradients():
    a = torch.randn(4, 5, device="cuda", dtype=torch.float64, requires_grad=True)
    b = torch.randn(5, 6, device="cuda", dtype=torch.float64)
    y = ome.ad_einsum(ome.ein("ij,jk->ik"), [a, b])
    y.sum().backward()
    assert b.grad is None and a.grad is not None
    assert torch.allclose(a.grad, torch.ones(4, 6, device="cuda", dtype=torch.float64) @ b.T)


GRAD_CODES = ["ij,jk->ik", "ij,jk,kl->il", "ijk,jkl->il", "ii->i", "ij,ij->", "ab,bc->acc", "ij->ji"]


@pytest.mark.parametrize("dt", ["f64", "c128", "f32", "c64", "i64", "trop"])
@pytest.mark.parametrize("code", GRAD_CODES)
def test_einsum_grad_matches_oracle(code, dt):
    """einsum_grad (one ome_einsum_grad call per input) against the oracle's
    restatement of src/autodiff.jl:24-30, for every input of the code."""
    import zlib
    import ome_oracle as O
    from helpers import assert_match, gen, parse, to_dev, to_np
    rng = np.random.default_rng(zlib.crc32(code.encode()) % 1000)
    ixs, iy = parse(code)
    sd = {l: 3 + (ord(l) % 3) for l in set("".join("".join(ix) for ix in ixs))}
    xs = [gen(rng, [sd[l] for l in ix], dt) for ix in ixs]
    dy = gen(rng, [sd[l] for l in iy], dt)
    alg = O.TROPICAL if dt == "trop" else None
    dxs = [to_dev(x, dt) for x in xs]
    for i in range(len(xs)):
        got = to_np(ome.einsum_grad(ixs, dxs, iy, sd, to_dev(dy, dt), i))
        want = O.einsum_grad(ixs, xs, iy, sd, dy, i, alg)
        assert_match(got, want, dt)


@pytest.mark.parametrize("dtype", [torch.float64, torch.complex128])
@pytest.mark.parametrize("code", ["ij,jk->ik", "ij,jk,kl->il", "ijk,jkl->il", "ij,ij->"])
def test_ad_einsum_gradients_match_oracle(code, dtype):
    """torch.autograd through ad_einsum: the gradients equal the oracle's
    einsum_grad with the cotangent torch hands the pullback (here the weight
    of a linear loss)."""
    import ome_oracle as O
    g = torch.Generator().manual_seed(5)
    lhs, iy = code.split("->")
    ixs = lhs.split(",")
    sd = {l: 3 + (ord(l) % 3) for l in set("".join(ixs))}
    xs_h = [torch.randn([sd[l] for l in ix], generator=g, dtype=torch.float64) for ix in ixs]
    if dtype.is_complex:
        xs_h = [x + 1j * torch.randn(x.shape, generator=g, dtype=torch.float64) for x in xs_h]
    w = torch.randn([sd[l] for l in iy], generator=g, dtype=torch.float64)
    dev_in = [x.to("cuda").requires_grad_(True) for x in xs_h]
    y = ome.ad_einsum(ome.EinCode([tuple(ix) for ix in ixs], tuple(iy)), dev_in)
    loss = (y * w.cuda()).real.sum() if y.is_complex() else (y * w.cuda()).sum()
    loss.backward()
    ome.device_status()
    xs_np = [x.numpy() for x in xs_h]
    dy = w.numpy().astype(np.complex128) if dtype.is_complex else w.numpy()
    for i, a in enumerate(dev_in):
        want = O.einsum_grad([tuple(ix) for ix in ixs], xs_np, tuple(iy), sd, dy, i)
        got = a.grad.detach().cpu().numpy()
        assert np.linalg.norm(got - want) <= 1e-10 * max(np.linalg.norm(want), 1e-300)
