"""The learned preconditioner's network on the GPU (rtkb_unet_*) against its
float64 torch-CPU oracle (oracle/unet_ref.py): forward pass, loss and every
layer's weight gradient, plus the training step itself.

The kernels store weights and activations in BF16 and accumulate in FP32; the
oracle rounds to BF16 at the same points and computes in FP64, so the
remaining differences are FP32 accumulation order, BF16 rounding of the
backward activations (the oracle keeps those in FP64) and rounding-boundary
flips.  Bounds: forward and loss within 1e-2 relative L2, gradients within
3e-2 per layer."""
import numpy as np
import pytest

from tests.gpu_util import rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-2
GRAD_TOL = 3e-2


def _net(seed=3):
    from rtk_b200.learned import UNet

    return UNet(seed=seed)


def _oracle_forward(x, flat, normalize=False):
    import torch

    from oracle import unet_ref

    ws = unet_ref.to_torch_weights(unet_ref.split(flat))
    with torch.no_grad():
        return unet_ref.forward(torch.as_tensor(x, dtype=torch.float64), ws, bf16=True,
                                normalize=normalize).numpy()


@pytest.mark.parametrize("shape", [(1, 16, 16, 16), (2, 12, 20, 24), (1, 8, 36, 20)])
def test_unet_forward_matches_oracle(rtkb, shape):
    net = _net()
    rng = np.random.default_rng(sum(shape))
    x = rng.standard_normal(shape).astype(np.float32)
    got = to_np(net.forward(to_gpu(x), normalize=False))
    ref = _oracle_forward(x.astype(np.float64), net.get_parameters())
    assert rel_l2(got, ref) < FWD_TOL, rel_l2(got, ref)
    net.close()


def test_unet_forward_normalized_is_homogeneous(rtkb):
    net = _net(5)
    rng = np.random.default_rng(11)
    x = rng.standard_normal((1, 16, 20, 24)).astype(np.float32) * 37.0
    g1 = to_np(net.forward(to_gpu(x), normalize=True))
    g2 = to_np(net.forward(to_gpu(x * 4.0), normalize=True))
    ref = _oracle_forward(x.astype(np.float64), net.get_parameters(), normalize=True)
    assert rel_l2(g1, ref) < FWD_TOL
    assert rel_l2(g2, 4.0 * g1) < 1e-6
    net.close()


@pytest.mark.parametrize("margin", [0, 3])
def test_unet_gradients_match_oracle(rtkb, margin):
    from oracle import unet_ref

    net = _net(7)
    rng = np.random.default_rng(5)
    shape = (2, 16, 12, 20)
    x = rng.standard_normal(shape).astype(np.float32)
    t = rng.standard_normal(shape).astype(np.float32) * 0.3
    params = net.get_parameters()
    loss = net.train_step(to_gpu(x), to_gpu(t), update=False, margin=margin)
    g = net.get_gradients()
    ref_loss, ref_g, _ = unet_ref.loss_and_gradients(x.astype(np.float64), t.astype(np.float64), params,
                                                     margin=margin)
    assert abs(loss - ref_loss) / ref_loss < FWD_TOL
    gl, rl = net.split(g), net.split(ref_g)
    for k, (a, b) in enumerate(zip(gl, rl)):
        assert rel_l2(a, b) < GRAD_TOL, (k, rel_l2(a, b))
    # no update: parameters unchanged
    assert np.array_equal(net.get_parameters(), params)
    net.close()


def test_unet_adam_step_matches_reference_update(rtkb):
    """One Adam step (lr 1e-3, bias-corrected) moves each weight by
    -lr * g / (|g| + eps) -- the first-step form of Adam."""
    net = _net(9)
    rng = np.random.default_rng(6)
    x = rng.standard_normal((1, 16, 16, 16)).astype(np.float32)
    t = rng.standard_normal((1, 16, 16, 16)).astype(np.float32) * 0.1
    p0 = net.get_parameters()
    net.train_step(to_gpu(x), to_gpu(t), lr=1e-3, update=True)
    g = net.get_gradients()
    p1 = net.get_parameters()
    expect = p0 - 1e-3 * g / (np.abs(g) + 1e-8)
    np.testing.assert_allclose(p1, expect, rtol=1e-4, atol=1e-7)
    net.close()


def test_unet_training_reduces_loss(rtkb):
    """A few hundred steps on a fixed smoothing target: the loss falls by at
    least 5x (the kernels' gradients point downhill)."""
    import torch

    net = _net(13)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0)
    x = torch.randn((4, 16, 16, 16), generator=gen, device="cuda")
    k = torch.ones((1, 1, 3, 3, 3), device="cuda") / 27.0
    t = torch.nn.functional.conv3d(x[:, None], k, padding=1)[:, 0].contiguous()
    first = net.train_step(x, t, lr=2e-3)
    for _ in range(300):
        last = net.train_step(x, t, lr=2e-3, want_loss=False)
    last = net.train_step(x, t, lr=1e-3)
    assert last < first / 5, (first, last)
    net.close()


def test_unet_rejects_sizes_not_multiple_of_4(rtkb):
    net = _net()
    with pytest.raises(rtkb.RtkbError):
        net.forward(to_gpu(np.zeros((1, 10, 16, 16), np.float32)))
    net.close()


@pytest.mark.parametrize("shape", [(2, 12, 20, 24), (1, 32, 32, 32)])
def test_unet_pipelined_convolution_equals_single_stage(rtkb, shape):
    """The convolution kernels with TMA halo and weight loads (one stage, the
    default, and two stages; zero fill outside the volume by the TMA unit,
    thread gathers for the up-sampled decoder inputs) issue the same MMAs in
    the same order as the thread-loaded kernel: the forward pass is
    bit-identical, and the training gradients (which add FP32 atomics in the
    weight gradient) agree to rounding."""
    lib = rtkb.load()
    net = _net(13)
    rng = np.random.default_rng(sum(shape) + 1)
    x = rng.standard_normal(shape).astype(np.float32)
    t = rng.standard_normal(shape).astype(np.float32) * 0.2
    out, grads = {}, {}
    try:
        for pipe in (1, 2, 0):
            assert lib.rtkb_unet_set_conv_pipeline(pipe) == 0
            out[pipe] = to_np(net.forward(to_gpu(x), normalize=False))
            net.train_step(to_gpu(x), to_gpu(t), update=False)
            grads[pipe] = net.get_gradients()
    finally:
        lib.rtkb_unet_set_conv_pipeline(1)
    for pipe in (1, 2):
        assert np.array_equal(out[0], out[pipe])
        assert rel_l2(grads[pipe], grads[0]) < 1e-5
    assert rtkb.ops.device_status() == 0
    net.close()


@pytest.mark.parametrize("kernel", [1, 2])
def test_unet_tcgen05_weight_gradient(rtkb, kernel):
    """The tcgen05 weight-gradient kernels (MN-major shared-memory operands:
    the halo's [k-half][voxel][8 channels] layout and the gradient tile as
    [channel group][voxel][8 channels]; output channels as M = 64 or 128,
    27 tap accumulators resident in tensor memory) give the warp-level
    kernel's gradients up to FP32 summation order, and the oracle's within
    the gradient bound."""
    from oracle import unet_ref

    lib = rtkb.load()
    net = _net(7)
    rng = np.random.default_rng(5)
    shape = (2, 16, 12, 20)
    x = rng.standard_normal(shape).astype(np.float32)
    t = rng.standard_normal(shape).astype(np.float32) * 0.3
    params = net.get_parameters()
    grads = {}
    try:
        for k in (0, kernel):
            assert lib.rtkb_unet_set_wgrad_kernel(k) == 0
            net.train_step(to_gpu(x), to_gpu(t), update=False)
            grads[k] = net.split(net.get_gradients())
    finally:
        lib.rtkb_unet_set_wgrad_kernel(0)
    assert rtkb.ops.device_status() == 0
    _, ref_g, _ = unet_ref.loss_and_gradients(x.astype(np.float64), t.astype(np.float64), params)
    for k, (a, b, r) in enumerate(zip(grads[kernel], grads[0], net.split(ref_g))):
        assert rel_l2(a, b) < 1e-5, (k, rel_l2(a, b))
        assert rel_l2(a, r) < GRAD_TOL, (k, rel_l2(a, r))
    with pytest.raises(rtkb.RtkbError):
        from rtk_b200._capi import check

        check(lib.rtkb_unet_set_wgrad_kernel(3))
    net.close()
