"""ctypes wrapper of the reference's own hot path built from its sources
(oracle/_ref/libtsr_ref.so, `make -C oracle ref`; test infrastructure only).

Tree::Tree(), Occupancy(tree) and Occupancy::extractCrust() of the reference
run on one thread over a scene's samples; their results come back through the
reference's own writers (Nodes/Leaves/DualCells/Occupancy::saveToFile) in
the reference's body layouts (Nodes.cpp:789-807, Leaves.cpp:261-292,
DualCells.cpp:378-385, Occupancy.cpp:722-766), parsed here.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_ref" / "libtsr_ref.so"
REFERENCE_SOURCES = Path("/root/reference/SurfaceReconstruction/SurfaceReconstruction")
_lib = None

DEFAULT_PARAMS = (2.0, 2.0, 100.0, 25.0, 1.0)   # App.cfg:64-70


def available() -> bool:
    return LIB_PATH.exists()


def build():
    subprocess.run(["make", "-s", "-C", str(_HERE), "ref"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        L.tsrr_last_error.restype = ctypes.c_char_p
        L.tsrr_run.argtypes = [ctypes.c_uint32, ctypes.c_uint32, P, P, P, P, P, ctypes.c_uint32, P, P, ctypes.c_int,
                               ctypes.c_int]
        L.tsrr_file.restype = ctypes.c_uint64
        L.tsrr_file.argtypes = [ctypes.c_char_p, P, ctypes.c_uint64]
        L.tsrr_samples.argtypes = [P, P, P, P, P, P]
        L.tsrr_occupancy.argtypes = [P]
        L.tsrr_mesh.argtypes = [P, P, P, P]
        L.tsrr_update.argtypes = [P, ctypes.c_uint32, ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _file(name):
    n = lib().tsrr_file(name.encode(), None, 0)
    buf = np.zeros(n, np.uint8)
    if n:
        lib().tsrr_file(name.encode(), _p(buf), n)
    return buf


SCOPE_DTYPE = np.dtype({"names": ["min", "size", "idx"], "formats": [("<f8", 3), "<f8", "<u4"],
                        "offsets": [0, 24, 32], "itemsize": 40})


def _fields():
    """The field the reference's Occupancy::saveToFile wrote, and
    getOccupancy of every leaf."""
    b = _file("ref.occupancy")
    c = b[:8].view(np.uint32)
    L, N = int(c[0]), int(c[1])
    o = 8
    f = {}
    for name in ("e_len", "e_sum", "s_len", "s_sum", "prior"):
        f[name] = b[o:o + 8 * L].view(np.float64).copy()
        o += 8 * L
    f["states"] = b[o:o + 4 * N].view(np.uint32).copy()
    o += 4 * N
    f["cone_count"] = float(b[o:o + 8].view(np.float64)[0])
    occ = np.zeros(L)
    lib().tsrr_occupancy(_p(occ))
    f["occ"] = occ
    return f


def update(samples, removal):
    """Occupancy::eraseSamples (removal) / addSamples of tree-order sample
    indices on the field of the last run; returns the updated field."""
    idx = np.ascontiguousarray(samples, np.uint32)
    if lib().tsrr_update(_p(idx), idx.shape[0], 1 if removal else 0) != 0:
        raise RuntimeError("reference update failed: " + lib().tsrr_last_error().decode())
    return _fields()


def run(scene, params=DEFAULT_PARAMS, stage=2, threads=1, outputs=True):
    """The reference's tree (stage 0), field (1) and raw DMC mesh (2) of a
    scene on `threads` OpenMP threads (1 for parity: the reference's
    single-thread order).  Returns a dict of numpy arrays (nothing with
    outputs=False, for timing)."""
    pos = np.ascontiguousarray(scene.pos, np.float64)
    nrm = np.ascontiguousarray(scene.nrm, np.float64)
    sc = np.ascontiguousarray(scene.scale, np.float64)
    cf = np.ascontiguousarray(scene.conf, np.float64)
    links = np.ascontiguousarray(scene.links, np.uint32)
    cams = np.ascontiguousarray(scene.cams, np.float64)
    prm = np.ascontiguousarray(params, np.float64)
    n, k = pos.shape[0], links.shape[1]
    if lib().tsrr_run(n, k, _p(pos), _p(nrm), _p(sc), _p(cf), _p(links), cams.shape[0], _p(cams), _p(prm),
                      stage, threads) != 0:
        raise RuntimeError("reference run failed: " + lib().tsrr_last_error().decode())
    if not outputs:
        return None
    out = {}
    b = _file("ref.nodes")
    nn = int(b[:4].view(np.uint32)[0])
    a = b[4:4 + 16 * nn].view(np.uint32).reshape(4, nn)
    out.update(children=a[0].copy(), parents=a[1].copy(), counts=a[2].copy(), starts=a[3].copy())
    b = _file("ref.leaves")
    cnt = b[:12].view(np.uint32)
    nn2, nl, ne = int(cnt[0]), int(cnt[1]), int(cnt[2])
    o = 12
    out["node_to_leaf"] = b[o:o + 4 * nn2].view(np.uint32).copy(); o += 4 * nn2
    s = b[o:o + 40 * nl].view(SCOPE_DTYPE); o += 40 * nl
    out["scopes"] = np.concatenate([s["min"], s["size"][:, None]], 1)
    out["node_idx"] = s["idx"].copy()
    out["nb_offsets"] = b[o:o + 4 * (nl + 1)].view(np.uint32).copy(); o += 4 * (nl + 1)
    out["nbs"] = b[o:o + 4 * ne].view(np.uint32).copy()
    b = _file("ref.dualCells")
    ni = int(b[:4].view(np.uint32)[0])
    out["dual_cells"] = b[4:4 + 4 * ni].view(np.uint32).reshape(-1, 8).copy()
    sp, sn = np.zeros((n, 3)), np.zeros((n, 3))
    ss, scf = np.zeros(n), np.zeros(n)
    sl, tg = np.zeros((n, k), np.uint32), np.zeros(n, np.uint32)
    lib().tsrr_samples(_p(sp), _p(sn), _p(ss), _p(scf), _p(sl), _p(tg))
    out.update(samples_pos=sp, samples_nrm=sn, samples_scale=ss, samples_conf=scf, samples_links=sl,
               permutation=tg)
    if stage >= 1:
        out["fields"] = _fields()
    if stage >= 2:
        c = np.zeros(2, np.uint32)
        lib().tsrr_mesh(_p(c), None, None, None)
        vp, vs, tr = np.zeros((int(c[0]), 3)), np.zeros(int(c[0])), np.zeros((int(c[1]), 3), np.uint32)
        lib().tsrr_mesh(_p(c), _p(vp), _p(vs), _p(tr))
        out.update(vpos=vp, vscale=vs, tris=tr)
    return out
