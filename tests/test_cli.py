"""The `mirorr` command line (mirorr_b200/cli): NIfTI-1 and ITK transform-file
I/O, option handling, and (GPU) a registration run equal to the library call.

NIfTI files are written here by a small independent writer; the reader must
turn their qform / sform / pixdim into ITK's LPS geometry:
voxel-to-RAS from the qform (qform_code > 0), else the sform, else pixdim;
spacing = column norms, direction = normalised columns, first two rows of
direction and origin negated.
"""
import gzip
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "mirorr_b200", "bin", "mirorr")


@pytest.fixture(scope="module")
def cli():
    from mirorr_b200 import build as mb_build
    mb_build.build()
    return mb_build.build_cli()


def write_nifti(path, data_zyx, qform=None, sform=None, pixdim=(1.0, 1.0, 1.0), qfac=1.0,
                dtype=np.float32, slope=1.0, inter=0.0):
    """Minimal NIfTI-1 writer: qform = (b, c, d, qx, qy, qz), sform = 3x4 rows."""
    nz, ny, nx = data_zyx.shape
    codes = {np.float32: (16, 32), np.int16: (4, 16), np.uint8: (2, 8)}
    dt, bp = codes[dtype]
    h = bytearray(352)
    struct.pack_into("<i", h, 0, 348)
    struct.pack_into("<8h", h, 40, 3, nx, ny, nz, 1, 1, 1, 1)
    struct.pack_into("<hh", h, 70, dt, bp)
    struct.pack_into("<8f", h, 76, qfac, *pixdim, 0, 0, 0, 0)
    struct.pack_into("<fff", h, 108, 352.0, slope, inter)
    struct.pack_into("<hh", h, 252, 1 if qform else 0, 1 if sform is not None else 0)
    if qform:
        struct.pack_into("<6f", h, 256, *qform)
    if sform is not None:
        for r in range(3):
            struct.pack_into("<4f", h, 280 + 16 * r, *sform[r])
    h[344:348] = b"n+1\0"
    raw = bytes(h) + np.ascontiguousarray(data_zyx.astype(dtype)).tobytes()
    if path.endswith(".gz"):
        with gzip.open(path, "wb") as f:
            f.write(raw)
    else:
        with open(path, "wb") as f:
            f.write(raw)


def info(cli, path):
    out = subprocess.run([cli, "--info", path], capture_output=True, text=True, check=True).stdout
    d = {}
    for line in out.splitlines():
        k, *v = line.split()
        d[k] = np.array([float(x) for x in v])
    return d


def lps_from_ras(A, t):
    sp = np.linalg.norm(A, axis=0)
    D = A / sp
    flip = np.diag([-1.0, -1.0, 1.0])
    return sp, flip @ D, flip @ t


def quat_matrix(b, c, d):
    a = np.sqrt(max(0.0, 1.0 - (b * b + c * c + d * d)))
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a + c * c - b * b - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a + d * d - b * b - c * c]])


def test_help_and_errors(cli, tmp_path):
    assert subprocess.run([cli, "--help"], capture_output=True).returncode == 0
    r = subprocess.run([cli, "--bogus", "x"], capture_output=True, text=True)
    assert r.returncode == 1 and "unknown option" in r.stderr
    img = tmp_path / "a.nii"
    write_nifti(str(img), np.zeros((4, 5, 6), np.float32))
    r = subprocess.run([cli, "-m", str(img), "-f", str(img), "--reorient-fixed"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "not available" in r.stderr
    r = subprocess.run([cli, "-m", str(img), "-f", str(img), "--crop", "4"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "movingX,movingY,fixedX,fixedY" in r.stderr
    r = subprocess.run([cli, "-m", str(img), "-f", str(img), "--blockmetric", "mi"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "nc" in r.stderr


@pytest.mark.parametrize("gz", [False, True])
def test_nifti_qform_geometry(cli, tmp_path, gz):
    rng = np.random.default_rng(1)
    data = rng.random((7, 6, 5)).astype(np.float32)
    b, c, d = 0.1, -0.2, 0.05
    q = (b, c, d, 10.5, -3.25, 7.0)
    pix = (0.8, 1.2, 2.0)
    path = str(tmp_path / ("q.nii.gz" if gz else "q.nii"))
    write_nifti(path, data, qform=q, pixdim=pix, qfac=-1.0)
    g = info(cli, path)
    R = quat_matrix(np.float32(b), np.float32(c), np.float32(d))
    A = R @ np.diag([np.float32(pix[0]), np.float32(pix[1]), -np.float32(pix[2])])
    sp, D, o = lps_from_ras(A, np.array(q[3:], np.float32).astype(np.float64))
    np.testing.assert_array_equal(g["size"], [5, 6, 7])
    np.testing.assert_allclose(g["spacing"], sp, rtol=1e-6)
    np.testing.assert_allclose(g["origin"], o, atol=1e-5)
    np.testing.assert_allclose(g["direction"].reshape(3, 3), D, atol=1e-6)
    assert abs(g["sum"][0] - float(data.astype(np.float64).sum())) < 1e-3


def test_nifti_sform_and_scaling(cli, tmp_path):
    data = (np.arange(4 * 5 * 6).reshape(4, 5, 6) % 100).astype(np.int16)
    S = np.array([[0.0, 1.5, 0.0, 4.0], [-0.9, 0.0, 0.0, 2.0], [0.0, 0.0, 1.1, -6.0]])
    path = str(tmp_path / "s.nii")
    write_nifti(path, data, sform=S, dtype=np.int16, slope=0.5, inter=1.0)
    g = info(cli, path)
    sp, D, o = lps_from_ras(S[:, :3].astype(np.float32).astype(np.float64),
                            S[:, 3].astype(np.float32).astype(np.float64))
    np.testing.assert_allclose(g["spacing"], sp, rtol=1e-6)
    np.testing.assert_allclose(g["origin"], o, atol=1e-6)
    np.testing.assert_allclose(g["direction"].reshape(3, 3), D, atol=1e-6)
    assert abs(g["sum"][0] - float((data.astype(np.float64) * 0.5 + 1.0).sum())) < 1e-3


def _tfm(path, kind, params, center):
    name = "Euler3DTransform_double_3_3" if kind == "rigid" else "AffineTransform_double_3_3"
    with open(path, "w") as f:
        f.write("#Insight Transform File V1.0\n#Transform 0\n")
        f.write(f"Transform: {name}\nParameters: {' '.join(repr(float(p)) for p in params)}\n")
        f.write(f"FixedParameters: {' '.join(repr(float(c)) for c in center)}\n")


def _read_tfm(path):
    d = {}
    for line in open(path):
        if ":" in line and not line.startswith("#"):
            k, v = line.split(":", 1)
            d[k.strip()] = v.split()
    return d


@pytest.mark.parametrize("kind", ["rigid", "affine"])
def test_tfm_round_trip_and_inverse(cli, tmp_path, kind):
    from oracle import oracle as O
    img = str(tmp_path / "a.nii")
    write_nifti(img, np.zeros((4, 5, 6), np.float32))
    params = ([0.05, -0.02, 0.1, 3.0, -1.5, 2.25] if kind == "rigid" else
              [1.02, 0.03, -0.01, 0.02, 0.97, 0.04, -0.03, 0.01, 1.05, 3.0, -1.5, 2.25])
    center = [1.5, -2.0, 0.5]
    src = str(tmp_path / "in.tfm")
    _tfm(src, kind, params, center)
    out = str(tmp_path / "out.tfm")
    subprocess.run([cli, "-R", "-q", "-t", kind, "-m", img, "-f", img, "-s", src, "-l", out],
                   check=True)
    d = _read_tfm(out)
    assert d["Transform"][0].startswith("Euler3D" if kind == "rigid" else "Affine")
    np.testing.assert_allclose([float(v) for v in d["Parameters"]], params, rtol=0, atol=1e-15)
    np.testing.assert_allclose([float(v) for v in d["FixedParameters"]], center, atol=0)
    inv = str(tmp_path / "inv.tfm")
    subprocess.run([cli, "-R", "-q", "-I", "-t", kind, "-m", img, "-f", img, "-s", src, "-l", inv],
                   check=True)
    t = O.Tfm(kind)
    t.set_center(center)
    t.set_params(params)
    ti = t.inverse()
    di = _read_tfm(inv)
    np.testing.assert_allclose([float(v) for v in di["Parameters"]], ti.params(), atol=1e-12)


@pytest.mark.gpu
def test_cli_registration_matches_library(cli, tmp_path):
    import mirorr_b200 as mb
    from mirorr_b200.phantom import make_phantom
    ph = make_phantom((48, 44, 40), n_gauss=12, kind="rigid", seed=31, max_angle_deg=4.0,
                      max_shift_vox=3.0)
    fix, mov = str(tmp_path / "fix.nii.gz"), str(tmp_path / "mov.nii.gz")
    write_nifti(fix, ph.fixed)
    write_nifti(mov, ph.moving)
    out = str(tmp_path / "r.tfm")
    res = str(tmp_path / "res.nii")
    subprocess.run([cli, "-q", "-m", mov, "-f", fix, "-l", out, "-t", "rigid", "-d", "2", "-c", "0",
                    "-n", "3", "--save-resampled-moving", res, "--final-interpolator", "linear"],
                   check=True)
    # the same registration through the library, on the geometry the reader
    # gives these files (no qform / sform: pixdim spacing, LPS-flipped axes)
    gf, gm = info(cli, fix), info(cli, mov)
    geom = lambda g: mb.Geometry.make(g["size"].astype(int), g["spacing"], g["origin"],  # noqa: E731
                                      g["direction"].reshape(3, 3))
    ctx = mb.Context(0)
    p = mb.reg_params(symmetric=True, kind="rigid", levels=2, iterations=3)
    # the command line registers the images reoriented to ARI
    fa, gfa = _ari_geometry(mb, ph.fixed, gf)
    ma, gma = _ari_geometry(mb, ph.moving, gm)
    t, _ = mb.register(ctx, fa, ma, p, gfa, gma)
    d = _read_tfm(out)
    np.testing.assert_allclose([float(v) for v in d["Parameters"]], t.param_vector(), rtol=0,
                               atol=1e-12)
    np.testing.assert_allclose([float(v) for v in d["FixedParameters"]], np.array(t.center),
                               atol=1e-12)
    # the resampled moving image: the library's linear resampling through T^-1
    from oracle import oracle as O
    tt = O.Tfm("rigid")
    tt.set_center(np.array(t.center))
    tt.set_params(t.param_vector())
    ti = tt.inverse()
    C, e = mb.resample_map(geom(gf), geom(gm), ti.M, ti.off)
    want, _ = mb.resample(ctx, ph.moving, None, gf["size"].astype(int), C, e)
    g = info(cli, res)
    np.testing.assert_array_equal(g["size"], [48, 44, 40])
    assert abs(g["sum"][0] - float(want.astype(np.float64).sum())) < 1e-2
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("interp", ["bspline", "sinc", "default"])
def test_cli_final_interpolators(cli, tmp_path, interp):
    # resample only (-R) through a given transform with the B-spline (the
    # reference's default) or windowed-sinc interpolator
    import mirorr_b200 as mb
    from oracle import oracle as O
    rng = np.random.default_rng(5)
    img = (rng.random((14, 15, 16)) * 50).astype(np.float32)
    src = str(tmp_path / "m.nii")
    write_nifti(src, img)
    tf = str(tmp_path / "t.tfm")
    params = [0.04, -0.03, 0.02, 0.7, -0.4, 0.3]
    _tfm(tf, "rigid", params, [0.0, 0.0, 0.0])
    res = str(tmp_path / "r.nii")
    cmd = [cli, "-R", "-q", "-t", "rigid", "-m", src, "-f", src, "-s", tf,
           "-l", str(tmp_path / "o.tfm"), "--save-resampled-moving", res]
    if interp != "default":
        cmd += ["--final-interpolator", interp]
    subprocess.run(cmd, check=True)
    g = info(cli, src)
    geom = mb.Geometry.make(g["size"].astype(int), g["spacing"], g["origin"],
                            g["direction"].reshape(3, 3))
    t = O.Tfm("rigid")
    t.set_center([0.0, 0.0, 0.0])
    t.set_params(params)
    ti = t.inverse()
    C, e = mb.resample_map(geom, geom, ti.M, ti.off)
    want = mb.resample_final(mb.Context(0), img, g["size"].astype(int), C, e,
                             "sinc" if interp == "sinc" else "bspline")
    assert abs(info(cli, res)["sum"][0] - float(want.astype(np.float64).sum())) < 1e-2


def _ari_of(data_zyx, D, origin, spacing):
    """Expected ARI reorientation: axis 0 along +y, 1 along +x, 2 along +z
    (LPS), each voxel keeping its physical position."""
    D = np.asarray(D, float)
    dom = [int(np.argmax(np.abs(D[:, c]))) for c in range(3)]
    p = [dom.index(t) for t in (1, 0, 2)]
    f = [1 if D[dom[c], c] > 0 else -1 for c in p]
    a = np.transpose(data_zyx, (2, 1, 0))  # (x, y, z) = axes 0, 1, 2
    a = np.transpose(a, p)
    for k in range(3):
        if f[k] < 0:
            a = np.flip(a, axis=k)
    n = data_zyx.shape[::-1]
    first_old = [0 if f[p.index(c)] > 0 else n[c] - 1 for c in range(3)]
    org = np.asarray(origin, float) + D @ (np.asarray(spacing, float) * first_old)
    Dn = np.stack([f[k] * D[:, p[k]] for k in range(3)], axis=1)
    return np.transpose(a, (2, 1, 0)), org, Dn, [n[c] for c in p]


def _ari_geometry(mb, data_zyx, g):
    """The ARI-reoriented array and its library geometry for an --info record."""
    D = g["direction"].reshape(3, 3)
    arr, org, Dn, size = _ari_of(data_zyx, D, g["origin"], g["spacing"])
    dom = [int(np.argmax(np.abs(D[:, c]))) for c in range(3)]
    sp = [g["spacing"][dom.index(t)] for t in (1, 0, 2)]
    return np.ascontiguousarray(arr), mb.Geometry.make(np.array(size), sp, org, Dn)


@pytest.mark.parametrize("perm", [(0, 1, 2), (1, 0, 2), (2, 0, 1)])
def test_ari_reorientation_geometry(cli, tmp_path, perm):
    rng = np.random.default_rng(3)
    data = rng.random((5, 6, 7)).astype(np.float32)
    # sform (RAS): axis c along RAS axis perm[c], alternating signs
    S = np.zeros((3, 4))
    sp = [0.9, 1.2, 1.5]
    for c in range(3):
        S[perm[c], c] = sp[c] * (1 if c % 2 == 0 else -1)
    S[:, 3] = [3.0, -2.0, 5.5]
    path = str(tmp_path / "o.nii")
    write_nifti(path, data, sform=S)
    g = info(cli, path)
    D = g["direction"].reshape(3, 3)
    want, org, Dn, size = _ari_of(data, D, g["origin"], g["spacing"])
    np.testing.assert_array_equal(g["ari_size"], size)
    np.testing.assert_allclose(g["ari_direction"].reshape(3, 3), Dn, atol=1e-9)
    np.testing.assert_allclose(np.abs(g["ari_direction"].reshape(3, 3)),
                               [[0, 1, 0], [1, 0, 0], [0, 0, 1]], atol=1e-9)
    np.testing.assert_allclose(g["ari_origin"], org, atol=1e-6)
    np.testing.assert_allclose(g["ari_first"], [want[0, 0, 0], want[-1, -1, -1]], rtol=1e-7)


@pytest.mark.gpu
def test_cli_registration_independent_of_storage_orientation(cli, tmp_path):
    # the same physical images stored in two voxel orders register alike: the
    # registration sees both reoriented to ARI
    from mirorr_b200.phantom import make_phantom
    ph = make_phantom((40, 36, 32), n_gauss=12, kind="rigid", seed=17, max_angle_deg=4.0,
                      max_shift_vox=3.0)
    outs = []
    for storage in ("ras", "ari"):
        if storage == "ras":
            S = np.array([[1.0, 0, 0, 2.0], [0, 1.0, 0, -3.0], [0, 0, 1.0, 1.0]])
            fix_d, mov_d = ph.fixed, ph.moving
        else:
            # the ARI voxel order of the RAS-stored images, with its sform
            D = np.diag([-1.0, -1.0, 1.0])
            fix_d, org, Dn, _ = _ari_of(ph.fixed, D, np.array([-2.0, 3.0, 1.0]), [1, 1, 1])
            mov_d, _, _, _ = _ari_of(ph.moving, D, np.array([-2.0, 3.0, 1.0]), [1, 1, 1])
            flip = np.diag([-1.0, -1.0, 1.0])
            S = np.concatenate([flip @ Dn, (flip @ org)[:, None]], axis=1)
        fix, mov = str(tmp_path / f"f_{storage}.nii"), str(tmp_path / f"m_{storage}.nii")
        write_nifti(fix, np.ascontiguousarray(fix_d), sform=S)
        write_nifti(mov, np.ascontiguousarray(mov_d), sform=S)
        out = str(tmp_path / f"{storage}.tfm")
        subprocess.run([cli, "-q", "-m", mov, "-f", fix, "-l", out, "-t", "rigid", "-d", "2",
                        "-c", "0", "-n", "3"], check=True)
        outs.append(np.array([float(v) for v in _read_tfm(out)["Parameters"]]))
    np.testing.assert_allclose(outs[0], outs[1], atol=1e-6)
