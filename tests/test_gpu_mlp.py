"""Warm-start network kernels on the tcgen05 tensor cores: the BF16 GEMM
against a float64 product of the same BF16 values (FP32 accumulation: 2e-5 of
the row scale)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> BF16 bit patterns."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_value(bits: np.ndarray) -> np.ndarray:
    return (bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


@pytest.fixture(scope="module")
def lib():
    from aerocfd_b200 import _lib, build
    build.build()
    return _lib.load()


@pytest.mark.parametrize("M,N,K,splits", [(128, 128, 64, 1), (256, 384, 192, 1), (128, 256, 1024, 4), (384, 128, 640, 3),
                                          (256, 1024, 320, 1), (128, 1152, 256, 2)])
def test_tensor_core_gemm(lib, M, N, K, splits):
    rng = np.random.default_rng(M + N + K)
    a = bf16_bits(rng.standard_normal((M, K)))
    b = bf16_bits(rng.standard_normal((N, K)))
    c = np.zeros((M, N), dtype=np.float32)
    p = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    rc = lib.aero_mlp_gemm(p(a), p(b), p(c), M, N, K, splits)
    assert rc == 0, lib.aero_last_error()
    ref = bf16_value(a) @ bf16_value(b).T
    scale = np.sqrt(K) * 4.0
    err = np.max(np.abs(c - ref)) / scale
    print("max abs err / scale", err)
    assert err < 2e-5


def _net(lib, n_in, n_out, width, depth, batch, seed=11):
    assert lib.aero_mlp_create(n_in, n_out, width, depth, batch, ctypes.c_ulonglong(seed)) == 0, lib.aero_last_error()
    cnt = ctypes.c_longlong(0)
    assert lib.aero_mlp_param_count(ctypes.byref(cnt)) == 0
    params = np.zeros(cnt.value, dtype=np.float32)
    assert lib.aero_mlp_get_params(params.ctypes.data_as(ctypes.c_void_p)) == 0
    return params


def test_gradients_match_float64_oracle(lib):
    import mlp_reference as R
    n_in, n_out, width, depth, batch = 5, 4, 128, 3, 512
    params = _net(lib, n_in, n_out, width, depth, batch)
    rng = np.random.default_rng(3)
    n = 400
    x = rng.uniform(-1, 1, (n, n_in)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) * x[:, 1], np.cos(x[:, 2]), x[:, 3] * x[:, 4], x[:, 0] ** 2], 1).astype(np.float32)
    loss = ctypes.c_float(0)
    grad = np.zeros_like(params)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.aero_mlp_gradients(p(x), p(t), n, ctypes.byref(loss), p(grad)) == 0, lib.aero_last_error()
    layers = R.unpack(params, 128, width, depth, 128)
    ref_loss, ref_grads, _ = R.loss_and_grads(layers, x.astype(np.float64), t.astype(np.float64))
    assert abs(loss.value - ref_loss) <= 1e-3 * ref_loss
    glayers = R.unpack(grad, 128, width, depth, 128)
    for l, ((gW, gb), (rW, rb)) in enumerate(zip(glayers, ref_grads)):
        ew = np.linalg.norm(gW - rW) / np.linalg.norm(rW)
        eb = np.linalg.norm(gb - rb) / np.linalg.norm(rb)
        print(f"layer {l}: |dW err| {ew:.2e}  |db err| {eb:.2e}")
        assert ew < 2e-2 and eb < 2e-2, (l, ew, eb)
    lib.aero_mlp_destroy()


def test_training_fits_and_predicts(lib):
    import mlp_reference as R
    n_in, n_out, width, depth, batch = 3, 2, 256, 4, 2048
    _net(lib, n_in, n_out, width, depth, batch, seed=5)
    rng = np.random.default_rng(8)
    n = 32768
    x = rng.uniform(-1, 1, (n, n_in)).astype(np.float32)
    t = np.stack([np.sin(3 * x[:, 0]) + x[:, 1] * x[:, 2], np.exp(-x[:, 0] ** 2 - x[:, 1] ** 2)], 1).astype(np.float32)
    steps = 600
    hist = np.zeros(steps, dtype=np.float32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.aero_mlp_train(p(x), p(t), ctypes.c_longlong(n), steps, ctypes.c_float(2e-3), ctypes.c_ulonglong(1),
                              p(hist)) == 0, lib.aero_last_error()
    print("loss first/last:", hist[:3], hist[-3:])
    assert np.all(np.isfinite(hist)) and hist[-20:].mean() < 0.05 * hist[:5].mean()
    y = np.zeros((n, n_out), dtype=np.float32)
    assert lib.aero_mlp_predict(p(x), ctypes.c_longlong(n), p(y)) == 0
    cnt = ctypes.c_longlong(0)
    lib.aero_mlp_param_count(ctypes.byref(cnt))
    params = np.zeros(cnt.value, dtype=np.float32)
    lib.aero_mlp_get_params(p(params))
    yr, _, _ = R.forward(R.unpack(params, 128, width, depth, 128), x[:4096].astype(np.float64))
    err = np.abs(y[:4096] - yr[:, :n_out]).max()
    print("predict vs float64 forward:", err)
    assert err < 2e-2
    assert np.mean((y - t) ** 2) < 0.05 * np.mean((t - t.mean(0)) ** 2)
    lib.aero_mlp_destroy()
