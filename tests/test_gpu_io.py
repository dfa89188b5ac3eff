"""NGA restart files straight from and to device memory
(dataReader.writeNGArestart_device / readNGArestart_device, the format of
src/data/dataReader.py:119-208): byte-identical to the serial host writer,
and read back bit for bit, with staging chunks small enough that every field
crosses several of them (and chunks that straddle variables)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("chunk", [8 * 1000, 8 * 4096, 1 << 26])
def test_device_restart_matches_host_format(tmp_path, chunk):
    import pyflow_b200.dataReader as dr
    rng = np.random.default_rng(3)
    shape = (24, 20, 28)
    host = [rng.standard_normal(shape) for _ in range(4)]
    names = ["U", "V", "W", "P"]
    dev = [torch.tensor(a, device="cuda") for a in host]
    f_dev, f_host = tmp_path / "dev.rst", tmp_path / "host.rst"
    dr.writeNGArestart_device(str(f_dev), dev, names, 0.005, 1.25, chunk_bytes=chunk)
    dr.writeNGArestart(str(f_host), host, names, 0.005, 1.25)
    assert f_dev.read_bytes() == f_host.read_bytes()
    nm, t, back = dr.readNGArestart_device(str(f_host), "cuda", chunk_bytes=chunk)
    assert nm == names and t == 1.25
    for a, b in zip(back, host):
        assert np.array_equal(a.cpu().numpy(), b)
    nm3, _, three = dr.readNGArestart_device(str(f_dev), "cuda", nvar=3, chunk_bytes=chunk)
    assert nm3 == names[:3] and len(three) == 3
    for a, b in zip(three, host):
        assert np.array_equal(a.cpu().numpy(), b)
