"""Field files in the reference's binary output format: the files this
project writes (dtfe_write_binary, dtfe_field_suffix through
dtfe_b200.output) equal, name for name and byte for byte, the ones the
reference's own writeBinaryFile / writeOutputData (compiled from its sources
in the harness) write for the same fields."""
import os

import numpy as np
import pytest

from dtfe_b200 import _native as N
from dtfe_b200 import output as OUT

NCOMP = {"density": 1, "velocity": 3, "velocity_gradient": 9, "velocity_divergence": 1, "velocity_shear": 5,
         "velocity_vorticity": 3, "velocity_std": 1, "scalar": 1, "scalar_gradient": 3}


def _ref():
    import refharness as R
    if not R.available():
        pytest.skip("reference harness not built (needs the reference tree)")
    return R


def _fields(rng, n, names):
    return {f: rng.standard_normal((n, NCOMP[f]) if NCOMP[f] > 1 else n).astype(np.float32) for f in names}


def test_write_binary_matches_reference(built, tmp_path):
    R = _ref()
    rng = np.random.default_rng(3)
    # 256^3 + 17 elements crosses the reference's write-block size
    for n, nc in ((256 ** 3 + 17, 1), (1000, 3), (777, 5), (513, 9), (0, 1)):
        a = rng.standard_normal((n, nc)).astype(np.float32)
        mine, ref = str(tmp_path / "mine.bin"), str(tmp_path / "ref.bin")
        OUT.write_binary(mine, a)
        R.write_binary(ref, a, nc)
        assert os.path.getsize(mine) == 4 * n * nc
        with open(mine, "rb") as f1, open(ref, "rb") as f2:
            assert f1.read() == f2.read(), (n, nc)


def test_write_fields_matches_write_output_data(built, tmp_path):
    R = _ref()
    rng = np.random.default_rng(4)
    n = 4321
    u = _fields(rng, n, [f for f in NCOMP if f != "velocity_std"])
    a = _fields(rng, n, list(NCOMP))
    mine = OUT.write_fields(str(tmp_path / "mine"), u) + OUT.write_fields(str(tmp_path / "mine"), a, averaged=True)
    R.write_output(str(tmp_path / "ref"), n, u, a)
    ref_files = sorted(p for p in os.listdir(tmp_path) if p.startswith("ref."))
    assert sorted(os.path.basename(p).replace("mine", "ref", 1) for p in mine) == ref_files
    assert len(ref_files) == 17
    for p in mine:
        q = os.path.join(tmp_path, os.path.basename(p).replace("mine", "ref", 1))
        with open(p, "rb") as f1, open(q, "rb") as f2:
            assert f1.read() == f2.read(), p


def test_suffixes_and_errors(built, tmp_path):
    assert OUT.suffix("density") == ".den" and OUT.suffix("density", averaged=True) == ".a_den"
    assert OUT.suffix("velocity_std") is None and OUT.suffix("velocity_std", averaged=True) == ".a_velStd"
    with pytest.raises(ValueError):
        OUT.write_fields(str(tmp_path / "x"), {"velocity_std": np.zeros(3, np.float32)})
    with pytest.raises(N.DTFEError) as e:
        OUT.write_binary(str(tmp_path / "no_such_dir" / "f.den"), np.zeros(4, np.float32))
    assert e.value.code == N.ERR_IO
