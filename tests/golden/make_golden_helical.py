"""Record the reference's own helical outputs (run on a machine with a GPU).

    python tests/golden/make_golden_helical.py OUTDIR

The reference's helical operators exist only as CUDA (XRecon
src/kernels/helical_arc3d.cu, bound at src/api/torch_binding.cpp:525-612).
oracle/build_oracle.py compiles that file unchanged, with the reference's
nvcc flags, into oracle/_ref/libxrecon_ref_helical.so behind a small C entry
(oracle/ref_helical_shim.cu).  This script runs the six operators through it
on seeded inputs and writes OUTDIR/helical_ref_<case>.npz, which are then
committed under tests/golden/ as the pin of the FP64 helical oracle.

Every output buffer is allocated with a zero guard band of one image plane
(or one detector) on both sides, and the script records whether the
reference wrote into it (``guard_ok``): its scatter kernels index the image
from FP32 guesses.  Images are square in x/y because the reference launches
its weighted backprojection with the x and y block counts swapped
(helical_arc3d.cu:1948-1951), which leaves voxels unwritten when W != H.
"""
from __future__ import annotations

import ctypes
import sys
import zlib
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

CASES = {
    # name: (options overrides, views, views per turn, flying focal spot)
    "one_turn_ffs": (dict(), 240, 96, True),
    "auto_tang": (dict(view_mode=0, weight_mode=1, tang_k=3.0, tang_blend=0.6, pitch=10.0, z0=-11.0), 200, 96,
                  False),
    "half_scan": (dict(view_mode=1, halfscan_coef=1.1, pitch=12.0, z0=-12.0), 180, 96, False),
}


def options(view_mode=2, weight_mode=0, view_turns=0.0, halfscan_coef=1.0, tang_k=5.0, tang_blend=0.0,
            pitch=8.0, z0=-9.0):
    """Packed options of HelicalProjector3d((32, 32, 16), (64, 8), (1.5, 1.5, 1.0), (3.0, 2.0), 300, 600,
    pixshift (0.2, -0.3, 0.25) voxels, binshift (0.25, -0.1) cells) with the given helical fields, and
    the source's rise per turn and start z."""
    du = 3.0 / 600.0
    o = [32, 32, 16, 64, 8, 1.5, 1.5, 1.0, du, 2.0, 300.0, 600.0, 0.2 * 1.5, -0.3 * 1.5, 0.25 * 1.0,
         0.25 * du, -0.1 * 2.0, 2, view_mode, weight_mode, view_turns, halfscan_coef, tang_k, tang_blend]
    return np.array(o, np.float32), float(pitch), float(z0)


def main(outdir: Path) -> None:
    from oracle import build_oracle
    so = build_oracle.REF_HELICAL_SO
    if not so.exists():
        raise SystemExit(f"{so} missing: build it with python oracle/build_oracle.py where the reference is present")
    lib = ctypes.CDLL(str(so))
    lib.xr_ref_helical.restype = ctypes.c_int
    lib.xr_ref_helical.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_float)] + [ctypes.c_void_p] * 4 + \
                                  [ctypes.c_int, ctypes.c_int]
    dev = torch.device("cuda:0")
    outdir.mkdir(parents=True, exist_ok=True)
    for name, (over, V, per_turn, ffs) in CASES.items():
        opts, pitch, z0 = options(**over)
        W, H, D, Nu, Nv = (int(v) for v in opts[:5])
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        ang = (np.arange(V) * (2 * np.pi / per_turn) + 0.05).astype(np.float32)
        sp = np.zeros((4, V), np.float32)
        sp[0] = (z0 + pitch * (ang.astype(np.float64) - ang[0]) / (2 * np.pi)).astype(np.float32)
        if ffs:
            sp[1] = rng.normal(0.0, 1.0, V)
            sp[2] = rng.normal(0.0, 5e-4, V)
            sp[3] = rng.normal(0.0, 0.3, V)
        x = rng.random((1, 1, D, H, W)).astype(np.float32)
        y = rng.random((1, 1, V, Nv, Nu)).astype(np.float32)
        nvox, ncell = D * H * W, V * Nv * Nu
        gi, gs = H * W, Nv * Nu  # guard bands
        img = torch.zeros(nvox + 2 * gi, device=dev)
        sino = torch.zeros(ncell + 2 * gs, device=dev)
        a = torch.from_numpy(ang).to(dev)
        s = torch.from_numpy(sp).to(dev)
        res = {}
        guard_ok = True
        hopts = (ctypes.c_float * 24)(*opts.tolist())
        for op, key, inp_is_img in ((0, "A", True), (1, "AT", False), (2, "B", False), (3, "BT", True),
                                    (4, "BW", False), (5, "BWT", True)):
            img.zero_()
            sino.zero_()
            if inp_is_img:
                img[gi:gi + nvox] = torch.from_numpy(x.reshape(-1)).to(dev)
            else:
                sino[gs:gs + ncell] = torch.from_numpy(y.reshape(-1)).to(dev)
            rc = lib.xr_ref_helical(op, hopts, img.data_ptr() + 4 * gi, sino.data_ptr() + 4 * gs, a.data_ptr(),
                                    s.data_ptr(), 1, V)
            if rc != 0:
                raise SystemExit(f"{name} {key}: CUDA error {rc}")
            if inp_is_img:
                out = sino[gs:gs + ncell].cpu().numpy().reshape(1, 1, V, Nv, Nu)
                guard_ok &= bool(sino[:gs].abs().max() == 0 and sino[gs + ncell:].abs().max() == 0)
            else:
                out = img[gi:gi + nvox].cpu().numpy().reshape(1, 1, D, H, W)
                guard_ok &= bool(img[:gi].abs().max() == 0 and img[gi + nvox:].abs().max() == 0)
            res[key] = out
        np.savez_compressed(outdir / f"helical_ref_{name}.npz", options=opts, angles=ang, source_pos=sp, image=x,
                            sino=y, guard_ok=np.bool_(guard_ok), **res)
        print(name, "guard_ok" if guard_ok else "GUARD WRITTEN", {k: float(np.abs(v).max()) for k, v in res.items()})


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
