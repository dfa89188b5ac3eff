"""Host-side packing of the MLP weights into the tensor-core operand layout
(K-major, no swizzle: 8-row x 16-byte core matrices, K chunks 128 B apart,
8-row groups 256 B apart).  Unpacking with the layout formula must give back
every BF16 weight and the float biases."""
import numpy as np
import torch


def test_pack_roundtrip():
    import pyflow_b200.sfsmodel_mlp as M
    p = M.xavier_init(1)
    p["b1"] = np.arange(128, dtype=np.float32)
    buf = M.pack(p)
    assert buf.size == 4096 + 32768 + 4096 + (128 + 128 + 16) * 4

    def unpack(base, rows, cols, sl):
        off = M._kmajor_offsets(rows, cols, sl) + base
        bits = buf[off].astype(np.uint16) | (buf[off + 1].astype(np.uint16) << 8)
        return torch.from_numpy(bits.view(np.int16).copy()).view(torch.bfloat16).float().numpy()

    bf = lambda a: torch.tensor(a).to(torch.bfloat16).float().numpy()
    W1 = unpack(0, 128, 16, 4096)
    assert np.array_equal(W1[:, :9], bf(p["W1"])) and not W1[:, 9:].any()
    assert np.array_equal(unpack(4096, 128, 128, 4096), bf(p["W2"]))
    W3 = unpack(4096 + 32768, 16, 128, 512)
    assert np.array_equal(W3[:6], bf(p["W3"])) and not W3[6:].any()
    bias = buf[40960:].view(np.float32)
    assert np.array_equal(bias[:128], p["b1"])
    # every byte of the three weight images is covered exactly once
    offs = np.concatenate([M._kmajor_offsets(128, 16, 4096).ravel(),
                           4096 + M._kmajor_offsets(128, 128, 4096).ravel(),
                           36864 + M._kmajor_offsets(16, 128, 512).ravel()])
    assert np.array_equal(np.sort(offs), np.arange(0, 40960, 2))


def test_xavier_bounds():
    import pyflow_b200.sfsmodel_mlp as M
    p = M.xavier_init(1)
    assert np.abs(p["W2"]).max() <= np.sqrt(6 / 256)
    assert np.abs(p["W1"]).max() <= np.sqrt(6 / 137)
    assert not p["b2"].any()
