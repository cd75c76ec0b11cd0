"""Seed profile files (ymgpu2d/main_ym.cu:179-217 format and interpolation)."""
import numpy as np
import pytest

from kh_simulations_b200.seed import SeedError, interpolate, load_profiles, read_seed, write_seed


def loop_interp(h, nx):
    """Scalar float32 transcription of main_ym.cu:200-206."""
    h = np.asarray(h, np.float32)
    nf = len(h)
    out = np.empty(nx)
    for i in range(nx):
        t = np.float32(np.float32(i) * np.float32(nf - 1)) / np.float32(nx - 1)
        t = np.float32(t)
        j = min(int(t), nf - 2)
        frc = np.float32(t - np.float32(j))
        out[i] = float(np.float32(h[j] * np.float32(np.float32(1.0) - frc)) + np.float32(h[j + 1] * frc))
    return out


def test_roundtrip_and_interpolation(tmp_path):
    rng = np.random.default_rng(5)
    prof = {k: rng.normal(size=37).astype(np.float32) for k in ("by", "ex", "ez", "az", "qA", "qB")}
    f = tmp_path / "s.bin"
    write_seed(f, prof)
    back = read_seed(f)
    for k in prof:
        assert np.array_equal(back[k], prof[k])
    for nx in (37, 64, 101, 768):
        got = load_profiles(f, nx)
        for k in prof:
            assert np.array_equal(got[k], loop_interp(prof[k], nx))
            assert got[k][0] == prof[k][0] and got[k][-1] == prof[k][-1]


def test_bad_files(tmp_path):
    f = tmp_path / "bad.bin"
    f.write_bytes(b"\x01\x00")
    with pytest.raises(SeedError):
        read_seed(f)
    write_seed(tmp_path / "ok.bin", {"by": np.zeros(8, np.float32)})
    data = (tmp_path / "ok.bin").read_bytes()
    (tmp_path / "trunc.bin").write_bytes(data[:-4])
    with pytest.raises(SeedError):
        read_seed(tmp_path / "trunc.bin")
    with pytest.raises(SeedError):
        interpolate(np.zeros(4, np.float32), 1)
