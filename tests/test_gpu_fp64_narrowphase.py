"""The opt-in FP64 narrowphase on the GPU: bit-identical to the oracle in the
same mode, orthonormal frames at FP64 accuracy, and per-scene: a batch that
mixes both modes gives each scene the bits it gets alone."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu


def _fp64(sc):
    sc.params["fp64_narrowphase"] = 1
    return sc


def test_fp64_mode_bit_identical_to_oracle(native, oracle_mod):
    for sc in (_fp64(scenes.random_cluster(2, n=60)), _fp64(scenes.settling_box(n_side=4)),
               _fp64(scenes.random_cluster(9, n=40, mu=0.0))):
        g = native.NativeScene.from_scene(sc)
        o = oracle_mod.OracleScene(sc)
        for _ in range(4):
            g.step(5)
            o.step(5)
            assert np.array_equal(g.state()[0], o.state()[0])
            assert np.array_equal(g.state()[1], o.state()[1])
            assert np.array_equal(g.gamma(), o.gamma())
        g.close()


def test_fp64_mode_frames_orthonormal(native):
    sc = _fp64(scenes.random_cluster(4, n=60))
    g = native.NativeScene.from_scene(sc)
    g.step(3)
    F = g.frames().reshape(-1, 3, 3)
    assert len(F) > 20
    gram = np.einsum("cij,ckj->cik", F, F)
    assert np.max(np.abs(gram - np.eye(3))) < 1e-15
    g.close()
    # parity mode keeps the reference's float normalisation
    g = native.NativeScene.from_scene(scenes.random_cluster(4, n=60))
    g.step(3)
    F = g.frames().reshape(-1, 3, 3)
    gram = np.einsum("cij,ckj->cik", F, F)
    assert np.max(np.abs(gram - np.eye(3))) > 1e-10
    g.close()


def test_batch_mixing_modes_identical_to_alone(native):
    scs = [scenes.random_cluster(1, n=40), _fp64(scenes.random_cluster(1, n=40)),
           _fp64(scenes.settling_box(n_side=4)), scenes.ball_on_ground(h=1e-3)]
    b = native.NativeBatch(scs)
    b.step(12)
    for i, sc in enumerate(scs):
        g = native.NativeScene.from_scene(sc)
        g.step(12)
        assert np.array_equal(b.state(i)[0], g.state()[0]), i
        assert np.array_equal(b.gamma(i), g.gamma()), i
        g.close()
    # the two copies of the same cluster differ only through the mode
    assert not np.array_equal(b.state(0)[0], b.state(1)[0])
