"""CPU tests of the synthetic workload generators (deterministic, right shapes and distributions)."""
import numpy as np

from distance_transform_benchmarks_b200 import workloads as wl


def test_config0_shape_and_determinism():
    a = wl.config0()
    b = wl.config0()
    assert a[0].shape == (512, 512) and a[0].dtype == np.uint8
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[2] == np.float32(np.float32(1) / np.float32(255) * np.float32(10))
    assert 5 <= int(a[1].sum()) <= 5 * 29  # 5 disks of radius 3 (29 px each, may overlap / clip)


def test_blob_noise_statistics():
    img = wl.blobs_gray(11, 512, 512, nblobs=0, noise=4.0)  # zero field + noise -> clipped normal
    assert img.max() <= 20 and img.mean() < 2.5


def test_maze_structure():
    img, (sx, sy) = wl.maze_gray(5, 256, 256)
    assert img[sy, sx] <= 8  # seed on a corridor
    walls = img >= 247
    assert 0.05 < walls.mean() < 0.3
    assert walls[0, :].all() and walls[:, 0].all()  # closed border


def test_voronoi_cells_and_noise():
    img = wl.voronoi_rgb(3, 300, 200, nsites=4, noise=0.0)
    colours = {tuple(c) for c in img.reshape(-1, 3)}
    assert len(colours) <= 4


def test_threads_do_not_change_pixels():
    import os, subprocess, sys
    code = "from distance_transform_benchmarks_b200 import workloads as wl; import hashlib; " \
           "print(hashlib.md5(wl.voronoi_rgb(9, 333, 222).tobytes() + wl.blobs_gray(9, 333, 222).tobytes()).hexdigest())"
    outs = set()
    for n in ("1", "5"):
        env = dict(os.environ, OMP_NUM_THREADS=n)
        outs.add(subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                                cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__)))).stdout)
    assert len(outs) == 1


def test_config3_specs():
    specs = wl.config3_specs()
    assert len(specs) == 1024
    assert all(64 <= w <= 2048 and 64 <= h <= 2048 for _, w, h, _, _ in specs)
    assert {g for _, _, _, g, _ in specs} == {np.float32(0.01), np.float32(0.1), np.float32(1.0)}
    assert [k for k, *_ in specs[:4]] == ["gray", "rgb8", "gray", "rgb8"]
    mpx = sum(w * h for _, w, h, _, _ in specs) / 1e6
    assert 250 < mpx < 450  # E[area] = 572.5^2 -> ~335 Mpx


def test_oracle_generator_build_gives_the_same_pixels():
    """bench.py's CPU reference arm makes its inputs with the oracle's build of the generators (so it loads no
    library of the package); both builds of csrc/datagen.cpp must give the same pixels."""
    import os, subprocess, sys
    code = ("import hashlib, sys; from distance_transform_benchmarks_b200 import workloads as wl\n"
            "if sys.argv[1] == 'oracle':\n"
            "    from oracle import oracle as orc; wl.use_generator(orc.workload_generator_path())\n"
            "specs = wl.config3_specs(n=6, smax=300)\n"
            "h = hashlib.md5()\n"
            "for s in specs:\n"
            "    img, mask, g = wl.make_image(s); h.update(img.tobytes()); h.update(mask.tobytes())\n"
            "h.update(wl.maze_gray(5, 200, 160)[0].tobytes())\n"
            "print(h.hexdigest())\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = [subprocess.run([sys.executable, "-c", code, which], capture_output=True, text=True, cwd=root, check=True)
            .stdout for which in ("package", "oracle")]
    assert outs[0] and outs[0] == outs[1]


def test_stratified_sample_mixes_kinds_and_sizes():
    specs = wl.config3_specs()
    idx = wl.stratified_indices(specs, 24.0)
    k = idx[1] - idx[0]
    assert k % 2 == 1 and idx == list(range(0, len(specs), k))
    kinds = {specs[i][0] for i in idx}
    assert kinds == {"gray", "rgb8"}
    mpx = sum(specs[i][1] * specs[i][2] for i in idx) / 1e6
    assert 10 < mpx < 60
