"""The trained-cloud writers (GaussianCloud.cpp:259-306, 414-443, 493-550),
packed on the device, against the reference's own writers on the same clouds.

* PLY: byte-identical (float fields copied, the same header).
* .splat: byte-identical except in records whose linear sigma or opacity
  comes from an exp that glibc's expf does not round correctly (the device
  rounds exp correctly; glibc differs in the last bit for ~0.06% of inputs).
* .spz: the gzip-decompressed stream identical except alpha bytes of such
  gaussians; equal streams give equal files (the same deflate settings and
  zlib).
The reference's tests (SplatTest.cpp:196-475) check these formats by
round-tripping its own reader; here the reference's writer is the oracle.
"""
from __future__ import annotations

import gzip
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle_lib as O
import parallax_b200 as px

pytestmark = pytest.mark.gpu

FORMATS = {"ply": 0, "splat": 1, "spz": 2}


def reference_bytes(cloud: px.GaussianCloud, fmt: str, fractional_bits: int = 12) -> bytes:
    """The reference writer's file, from oracle/_ref/ref_writer (its own process)."""
    tool = os.path.join(os.path.dirname(O.ref_path("ieee")), "ref_writer")
    with tempfile.TemporaryDirectory() as d:
        src, path = os.path.join(d, "cloud.f32"), os.path.join(d, "cloud." + fmt)
        np.ascontiguousarray(cloud.params, dtype=np.float32).tofile(src)
        subprocess.run([tool, src, str(cloud.count), str(cloud.rest_per_channel),
                        str(cloud.sh_degree), str(FORMATS[fmt]), str(fractional_bits), path],
                       check=True)
        return open(path, "rb").read()


def clouds():
    a, rest = O.random_cloud(61, 5000, 3, log_scale_mean=-3.0)
    b, rest0 = O.random_cloud(62, 3000, 0, log_scale_mean=-4.0)
    c, _ = O.random_cloud(63, 1000, 3, log_scale_mean=-2.0)
    # edges: far positions (past the 24-bit range at 12 fractional bits),
    # log sigma outside [-10, 6], quaternions with w < 0, saturated colours
    c[0:3, :50] *= 5000.0
    c[3:6, 50:100] = np.linspace(-14, 9, 150).reshape(3, 50)
    c[6, 100:200] *= -1.0
    c[11:14, 200:250] = np.linspace(-5, 5, 150).reshape(3, 50)
    return [px.GaussianCloud(a, 3, rest), px.GaussianCloud(b, 0, rest0),
            px.GaussianCloud(np.ascontiguousarray(c), 1, rest)]  # SH3 storage, degree 1


def exp_exact(cloud):
    p = cloud.params
    return O.glibc_exp_is_correctly_rounded(np.stack([p[3], p[4], p[5], -p[10]])).all(axis=0)


@pytest.mark.parametrize("k", range(3))
def test_ply_is_byte_identical(k):
    cloud = clouds()[k]
    assert px.export_cloud(cloud, "ply") == reference_bytes(cloud, "ply")


@pytest.mark.parametrize("k", range(3))
def test_splat_matches_but_for_glibc_exp(k):
    cloud = clouds()[k]
    ours = np.frombuffer(px.export_cloud(cloud, "splat"), np.uint8).reshape(-1, 32)
    ref = np.frombuffer(reference_bytes(cloud, "splat"), np.uint8).reshape(-1, 32)
    assert ours.shape == ref.shape == (cloud.count, 32)
    differ = (ours != ref).any(axis=1)
    assert not (differ & exp_exact(cloud)).any()
    assert differ.sum() <= max(3, cloud.count // 100)


@pytest.mark.parametrize("k", range(3))
@pytest.mark.parametrize("bits", [12, 8])
def test_spz_matches_but_for_glibc_exp(k, bits):
    cloud = clouds()[k]
    ours_file, ref_file = px.export_cloud(cloud, "spz", bits), reference_bytes(cloud, "spz", bits)
    ours, ref = gzip.decompress(ours_file), gzip.decompress(ref_file)
    assert len(ours) == len(ref)
    n = cloud.count
    alpha_at = 16 + n * (9 + 3 + 3)
    a = np.frombuffer(ours, np.uint8)
    b = np.frombuffer(ref, np.uint8)
    outside = np.ones(len(a), bool)
    outside[alpha_at:alpha_at + n] = False
    assert np.array_equal(a[outside], b[outside])  # header, positions, scales, rotations, colour, SH
    alpha_differs = a[alpha_at:alpha_at + n] != b[alpha_at:alpha_at + n]
    assert not (alpha_differs & exp_exact(cloud)).any()
    if ours == ref:
        assert ours_file == ref_file


def test_trainer_export_and_refusals():
    cloud = clouds()[0]
    views = O.orbit_views(2, 32, 24, seed=9)
    images = [np.zeros(32 * 24 * 3, np.float32) for _ in views]
    t = px.SplatTrainer(cloud, [(v.camera(), im) for v, im in zip(views, images)],
                        px.TrainConfig(iterations=5))
    for fmt in ("ply", "splat", "spz"):
        assert t.export(fmt) == px.export_cloud(px.GaussianCloud(t.cloud_params(), 3, 15), fmt)
    t.close()
    empty = px.GaussianCloud(np.zeros((59, 0), np.float32), 3, 15)
    with pytest.raises(px.PxsError):
        px.export_cloud(empty, "ply")
