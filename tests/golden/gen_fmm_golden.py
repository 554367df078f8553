"""Regenerate tests/golden/fmm_golden.npz from the reference's own fast
marching method (its C sources built by ``make -C oracle ref`` into
oracle/_ref/libfmm.so): computeDistanceFunction3d on seeded unions of spheres
(anisotropic spacing, with and without a mask, 3D and 2D), orders 1 and 2,
computeExtensionFields3d on the same cases with two seeded source fields
(and an extension mask in the masked case), and solveEikonalEquation3d with
the region phi <= 0 as boundary data (shifted as the reference's Python
wrapper does) and a seeded speed (a zero-speed wall in the masked case).

    make -C oracle ref && python tests/golden/gen_fmm_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fmm_golden.npz")


def cases():
    """(name, phi (nz, ny, nx), dx per axis (dz, dy, dx), mask or None)."""
    rng = np.random.default_rng(2024)
    out = []
    for name, shape, h, masked in (("spheres3d", (17, 19, 24), (0.09, 0.12, 0.1), False),
                                   ("masked3d", (15, 21, 18), (0.1, 0.1, 0.1), True),
                                   ("spheres2d", (1, 30, 40), (1.0, 0.07, 0.05), False)):
        axes = [(np.arange(n) + rng.uniform(0.1, 0.4)) * d for n, d in zip(shape, h)]
        z, y, x = np.meshgrid(*axes, indexing="ij")
        ext = [n * d for n, d in zip(shape, h)]
        phi = np.full(shape, np.inf)
        for _ in range(2):
            c = [rng.uniform(0.3, 0.7) * e for e in ext]
            r = rng.uniform(0.15, 0.3) * min(e for e, n in zip(ext, shape) if n > 1)
            phi = np.minimum(phi, np.sqrt((z - c[0]) ** 2 * (shape[0] > 1) + (y - c[1]) ** 2
                                          + (x - c[2]) ** 2) - r)
        mask = None
        if masked:
            mask = np.ones(shape)
            mask[:, :4, :5] = -1.0          # a corner outside the domain
        out.append((name, phi, h, mask))
    return out


def sources(name, phi, mask):
    """Two source fields (quantised to 1/64, so they compress) and, with a
    mask, an extension mask."""
    rng = np.random.default_rng(len(name) * 7919)
    src = [np.round(64 * rng.standard_normal(phi.shape)) / 64,
           np.round(64 * np.cos(0.37 * np.arange(phi.size, dtype=np.float64))).reshape(
               phi.shape) / 64]
    emask = None
    if mask is not None:
        emask = np.where(rng.random(phi.shape) < 0.3, -1.0, 1.0)
    return src, emask


def eikonal_case(name, phi, mask):
    """Boundary data (the reference Python wrapper's shift of phi) and speed."""
    minphi = phi.min()
    data = np.where(phi > 0, minphi - 1.0, phi) - minphi
    x = np.linspace(0.0, 1.0, phi.size).reshape(phi.shape)
    speed = np.round(64 * (1.0 + 0.5 * np.sin(40 * x))) / 64   # compresses
    if mask is not None:
        speed[:, 12:14, :] = 0.0          # a wall the front cannot cross
    return data, speed


def main():
    fmm = oracle.reference_fmm()
    ext = oracle.reference_extension()
    eik = oracle.reference_eikonal()
    blobs = {}
    for name, phi, h, mask in cases():
        blobs[name + "|phi"] = phi
        blobs[name + "|dx"] = np.array(h)
        if mask is not None:
            blobs[name + "|mask"] = mask
        src, emask = sources(name, phi, mask)
        for k, a in enumerate(src):
            blobs["%s|src%d" % (name, k)] = a
        if emask is not None:
            blobs[name + "|emask"] = emask
        for order in (1, 2):
            blobs["%s|out%d" % (name, order)] = fmm(phi, order, h[::-1], mask)
            dist, fields = ext(phi, src, order, h[::-1], mask, emask)
            # the distance of the extension call is the distance function's
            assert np.array_equal(dist.view(np.uint64),
                                  blobs["%s|out%d" % (name, order)].view(np.uint64))
            for k, f in enumerate(fields):
                blobs["%s|ext%d_%d" % (name, order, k)] = f
        data, speed = eikonal_case(name, phi, mask)    # recomputed by the tests
        for order in (1, 2):
            blobs["%s|eik%d" % (name, order)] = eik(data, speed, order, h[::-1], mask)
    np.savez_compressed(OUT, **blobs)
    print("wrote %s (%.1f KB)" % (OUT, os.path.getsize(OUT) / 1024))


if __name__ == "__main__":
    main()
