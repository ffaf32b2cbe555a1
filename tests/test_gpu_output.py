"""dtfe_gpu_write_binary_dev: device fields streamed to files in the
reference's binary output format equal the host writer's files (themselves
equal to the reference's writeBinaryFile, tests/test_output.py), across
chunk boundaries of the pinned staging and for an empty field."""
import numpy as np
import pytest

from dtfe_b200 import output as OUT

pytestmark = pytest.mark.gpu


def test_write_binary_dev(gpu_built, tmp_path):
    import torch
    from dtfe_b200.device import DeviceDTFE
    rng = np.random.default_rng(5)
    with DeviceDTFE(0) as d:
        # 3.2 chunks of 32 MB, one element, empty
        for n in (27_000_000, 1, 0):
            a = rng.standard_normal(n).astype(np.float32)
            t = torch.from_numpy(a).cuda()
            mine, host = str(tmp_path / "dev.den"), str(tmp_path / "host.den")
            d.write_binary_dev(mine, t)
            OUT.write_binary(host, a)
            with open(mine, "rb") as f1, open(host, "rb") as f2:
                assert f1.read() == f2.read(), n
        fields = {"density": torch.randn(1000, device="cuda"), "velocity_gradient": torch.randn(1000, 9, device="cuda")}
        paths = OUT.write_fields(str(tmp_path / "snap"), fields, averaged=True, device=d)
        assert [p.rsplit(".", 1)[1] for p in paths] == ["a_den", "a_velGrad"]
        for p, f in zip(paths, ["density", "velocity_gradient"]):
            assert np.array_equal(np.fromfile(p, np.float32), fields[f].cpu().numpy().ravel())


def test_write_binary_dev_unwritable(gpu_built, tmp_path):
    import torch
    from dtfe_b200 import _native as N
    from dtfe_b200.device import DeviceDTFE
    with DeviceDTFE(0) as d:
        with pytest.raises(N.DTFEError) as e:
            d.write_binary_dev(str(tmp_path / "missing_dir" / "x.den"), torch.zeros(100, device="cuda"))
        assert e.value.code == N.ERR_IO
        # the handle stays usable
        d.write_binary_dev(str(tmp_path / "ok.den"), torch.ones(100, device="cuda"))
        assert np.array_equal(np.fromfile(str(tmp_path / "ok.den"), np.float32), np.ones(100, np.float32))
