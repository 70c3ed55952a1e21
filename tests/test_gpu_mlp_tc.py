"""The fused tensor-core inference kernel of the proposal network
(flpr_mlp_infer: tcgen05.mma with accumulators in tensor memory, one launch
for every layer) against the layer-by-layer kernels (flpr_mlp_fwd) and the
CPU oracle, which applies the same BF16 roundings."""
import numpy as np
import pytest
import torch

from oracle import mlp as om

pytestmark = pytest.mark.gpu


def _lib():
    from fastlpr_b200 import _lib as L
    return L, L.load()


@pytest.mark.parametrize("dims,batch", [([416, 256, 256, 256, 1], 1),
                                        ([416, 256, 256, 256, 1], 37),
                                        ([416, 256, 256, 256, 1], 300),
                                        ([40, 256, 1], 129)])
def test_fused_inference_matches_layer_kernels_and_oracle(cuda_ok, dims, batch):
    from fastlpr_b200 import learned
    L, lib = _lib()
    nl = len(dims) - 1
    dims_c = L.ivec(dims)
    assert lib.flpr_mlp_infer_supported(nl, dims_c) == 1
    rng = np.random.default_rng(batch)
    params = learned.init_params(dims, seed=batch)
    params = params + 0.05 * rng.standard_normal(params.shape).astype(np.float32)
    x = rng.standard_normal((batch, dims[0])).astype(np.float32)
    s = torch.cuda.current_stream().cuda_stream
    p32 = torch.tensor(params, device="cuda")
    p16 = p32.to(torch.bfloat16)
    x16 = torch.tensor(x, device="cuda").to(torch.bfloat16)
    out = torch.full((batch,), float("nan"), dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.check(lib.flpr_mlp_infer(nl, dims_c, p16.data_ptr(), p32.data_ptr(), batch,
                               x16.data_ptr(), out.data_ptr(), status.data_ptr(), s),
            "flpr_mlp_infer")
    ref = torch.empty((batch, 1), dtype=torch.float32, device="cuda")
    ws = torch.empty(lib.flpr_mlp_ws(nl, dims_c, batch), dtype=torch.uint8, device="cuda")
    L.check(lib.flpr_mlp_fwd(nl, dims_c, p16.data_ptr(), p32.data_ptr(), batch, x16.data_ptr(),
                             ref.data_ptr(), ws.data_ptr(), ws.numel(), s), "flpr_mlp_fwd")
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    got = out.cpu().numpy()
    want = ref.cpu().numpy()[:, 0]
    assert np.all(np.isfinite(got))
    scale = np.max(np.abs(want)) + 1e-30
    # both accumulate in FP32 and round every hidden layer to BF16; their
    # summation orders differ, so a hidden value may round the other way
    assert np.max(np.abs(got - want)) / scale < 2e-2
    oracle_out, _ = om.forward(params, dims, x)
    assert np.max(np.abs(got - oracle_out[:, 0])) / scale < 2e-2


def test_fused_inference_rejects_other_shapes(cuda_ok):
    L, lib = _lib()
    for dims in ([416, 128, 1], [416, 256, 2], [500, 256, 1], [30, 256, 1]):
        assert lib.flpr_mlp_infer_supported(len(dims) - 1, L.ivec(dims)) == 0
        assert lib.flpr_mlp_infer(len(dims) - 1, L.ivec(dims), None, None, 1, None, None, None,
                                  None) == -1
