"""Generates the golden fixtures in this directory from the reference's own code.

Runs the reference's C++ classes (compiled from the reference tree by oracle/Makefile into
oracle/_ref/librzk_ref.so) on the seeded synthetic scenes and records their outputs:
BVH build products, primary-hit receivers, visibility of seeded segments, VPLs from the
counter-based stream, and gather images in all four clamp modes.  Large arrays are stored
as SHA-256 digests of their bytes plus a small sample; small ones in full.

    python tests/golden/make_golden.py      (needs the reference tree; run in the build
                                             container, commit the .npz files)
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from oracle import RefHarness  # noqa: E402
from renzoku_b200 import scenegen as sg  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def segments(n, seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.1, 1.1, (n, 3)).astype(np.float32)
    q = rng.uniform(-0.1, 1.1, (n, 3)).astype(np.float32)
    return p, q


SCENES = {
    "room_boxes_32": lambda: sg.room_boxes(32, 32),
    "room_objects_60": lambda: sg.room_objects(60, 24, 24),
}
VPL = {"room_boxes_32": (7, 512, 3), "room_objects_60": (11, 256, 6)}
TAU = {0: 0.0, 1: 1e-3, 2: 0.05, 3: 0.05}


def main():
    oracle.build(ref=True)
    for name, mk in SCENES.items():
        sc = mk()
        ref = RefHarness(sc)
        codes, perm, nodes = ref.bvh()
        cam = ref.camera()
        recv = ref.primary()
        p, q = segments(4096, 5)
        occ = ref.occluded(p, q)
        seed, npart, mb = VPL[name]
        vpls = ref.vpl_generate(seed, npart, mb)
        hit = recv[recv["mat"] >= 0]
        images = {}
        for mode, tau in TAU.items():
            images[f"gather_{mode}"] = ref.gather(hit, vpls[:128], mode, tau)
        out = dict(n_tris=ref.n_tris, n_nodes=ref.n_nodes, codes=codes, perm=perm,
                   nodes_sha=digest(nodes), nodes_head=nodes[:64].view(np.uint8),
                   camera=cam.view(np.uint8), recv=recv.view(np.uint8), recv_sha=digest(recv),
                   seg_p=p, seg_q=q, occluded=occ, vpl=vpls.view(np.uint8), vpl_sha=digest(vpls),
                   vpl_seed=seed, vpl_particles=npart, vpl_max_bounce=mb, **images)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, ref.n_tris, ref.n_nodes, len(vpls), {k: float(v.sum()) for k, v in images.items()})


def clustering():
    sys.path.insert(0, os.path.dirname(HERE))
    from cluster_inputs import small_matrix
    sc = sg.room_objects(120, 24, 24, seed_geo=31, seed_mat=32)
    ref = RefHarness(sc)
    mat = small_matrix()
    alphas, norms = ref.ltm_alphas(mat)
    c, r, w, a = ref.cluster_by_sampling(mat, 60, 77)
    np.savez_compressed(os.path.join(HERE, "clustering_small.npz"), matrix_sha=digest(mat), alphas=alphas,
                        norms=norms, center=c, rep=r, weight=w, assign=a, num_clusters=60, seed=77)
    print("clustering", len(c))


if __name__ == "__main__":
    main()
    clustering()
