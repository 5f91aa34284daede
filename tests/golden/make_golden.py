"""Writes the golden fixtures of tests/golden/ from the reference bml library
built from its own sources (oracle/_ref/libbml_ref.so, `make -C oracle`).

    python tests/golden/make_golden.py

Fixtures (numpy .npz):
  x2_chain.npz     chain Hamiltonian N=256 (bml_b200_gen_chain, seed 0, M=64);
                   the reference's X^2 at threshold 1e-5 with M2=128: value,
                   index, nnz of the product and the two traces.
  x2_random.npz    the reference's own random test matrix (srand(1),
                   bml_random_matrix(ellpack, double, 13, 13)), as used by
                   tests/C-tests/multiply_matrix_x2_typed.c, and its X^2 at
                   threshold 0.
  sp2_chain.npz    SP2 (the loop of bml_b200_sp2, 12 iterations, threshold
                   1e-5, occupation N/2) on the chain, run on the reference's
                   bml_multiply_x2 / bml_copy / bml_add: the density matrix.
  ellblock_x2.npz  ELLBLOCK random test matrix, block sizes (5+i)%6+1 over
                   N=24, and the dense form of its X^2 at threshold 0.
  generators.json  sha256 of the chain (N=4096, M=128) and 40^3 lattice
                   (radius 3, M=256) generator outputs, seed 0.
  hamiltonian600.npz  the reference's example Hamiltonian
                   (examples/example1/hamiltonian.dat: N=600, dense, read as
                   examples/example1/main.f90 reads it) imported by the
                   reference into ELLPACK at threshold 0.05 with M=64 (the
                   example converts at 0.05): value, index, nnz.  The tests
                   run the reference library itself on it for the products.
                   `python tests/golden/make_golden.py hamiltonian` writes
                   only this file (it needs the reference's source tree).
"""
import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bml_b200 as B  # noqa: E402  (generators only: host code, no GPU)
from oracle import oracle as O  # noqa: E402

libc = C.CDLL(None)


def main():
    lib = O.ref()
    # X^2 of the chain
    N, M, M2 = 256, 64, 128
    v, ix, nz = B.gen_chain(N, M, 0)
    X = O.ref_ellpack(v, ix, nz, N, M)
    X2 = lib.bml_zero_matrix(2, 2, N, M2, 0)
    tr = O.ref_x2(X, X2, 1e-5)
    a = O.ref_ellpack_arrays(X2)
    np.savez_compressed(os.path.join(HERE, "x2_chain.npz"), value=a[0], index=a[1], nnz=a[2], trace=tr,
                        N=N, M2=M2)
    # the reference test's random matrix
    libc.srand(1)
    R = lib.bml_random_matrix(2, 2, 13, 13, 0)
    r = O.ref_ellpack_arrays(R)
    R2 = lib.bml_zero_matrix(2, 2, 13, 13, 0)
    tr = O.ref_x2(R, R2, 0.0)
    r2 = O.ref_ellpack_arrays(R2)
    np.savez_compressed(os.path.join(HERE, "x2_random.npz"), value=r[0], index=r[1], nnz=r[2],
                        value2=r2[0], index2=r2[1], nnz2=r2[2], trace=tr)
    # SP2 on the chain with the reference's building blocks
    H = O.ref_ellpack(np.pad(v.reshape(N, M), ((0, 0), (0, M2 - M))).reshape(-1),
                      np.pad(ix.reshape(N, M), ((0, 0), (0, M2 - M))).reshape(-1), nz, N, M2)
    D = lib.bml_zero_matrix(2, 2, N, M2, 0)
    T = lib.bml_zero_matrix(2, 2, N, M2, 0)
    lib.bml_copy(H, D)
    b = lib.bml_gershgorin(H)
    bb = (C.c_double * 2).from_address(b)
    lib.bml_normalize(D, bb[0], bb[1])
    occ = N / 2.0
    for _ in range(12):
        t = O.ref_x2(D, T, 1e-5)
        if abs(t[1] - occ) <= abs(2 * t[0] - t[1] - occ):
            lib.bml_copy(T, D)
        else:
            lib.bml_add(D, T, 2.0, -1.0, 1e-5)
    d = O.ref_ellpack_arrays(D)
    np.savez_compressed(os.path.join(HERE, "sp2_chain.npz"), value=d[0], index=d[1], nnz=d[2], M=M2)
    # ELLBLOCK
    Nb = 24
    bs, cnt = [], 0
    for i in range(Nb):
        s = (5 + i) % 6 + 1
        if cnt + s > Nb:
            s = Nb - cnt
        bs.append(s)
        cnt += s
        if cnt == Nb:
            break
    arr = (C.c_int * len(bs))(*bs)
    lib.bml_set_block_sizes(arr, len(bs), len(bs))
    libc.srand(5)
    E = lib.bml_random_matrix(3, 2, Nb, Nb, 0)
    E2 = lib.bml_zero_matrix(3, 2, Nb, Nb, 0)
    p = lib.bml_multiply_x2(E, E2, 0.0)
    etr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(2,)).copy()
    es = C.cast(E, C.POINTER(O.EllblockStruct)).contents
    nbk, mbk = es.NB, es.MB
    indexb = np.ctypeslib.as_array(es.indexb, shape=(nbk * mbk,)).copy()
    nnzb = np.ctypeslib.as_array(es.nnzb, shape=(nbk,)).copy()
    np.savez_compressed(os.path.join(HERE, "ellblock_x2.npz"), bsize=np.array(bs), indexb=indexb, nnzb=nnzb,
                        MB=mbk, dense=O.ref_to_dense(E, Nb), dense2=O.ref_to_dense(E2, Nb), trace=etr)
    # generator digests
    dig = {}
    for name, (vv, ii, nn) in (("chain_4096_128", B.gen_chain(4096, 128, 0)),
                                ("lattice_40_r3_256", B.gen_lattice(40, 3, 64000, 256, 0))):
        h = hashlib.sha256()
        for arr_ in (vv, ii, nn):
            h.update(np.ascontiguousarray(arr_).tobytes())
        dig[name] = h.hexdigest()
    json.dump(dig, open(os.path.join(HERE, "generators.json"), "w"), indent=1)
    print("golden fixtures written")


def hamiltonian():
    ref_dir = os.environ.get("BML_REFERENCE_DIR", "/root/reference")
    raw = np.loadtxt(os.path.join(ref_dir, "examples", "example1", "hamiltonian.dat"))
    n = int(raw[0])
    H = np.ascontiguousarray(raw[1:].reshape(n, n))  # read(1,*) H(i,j), j fastest
    lib = O.ref()
    M = 64
    A = lib.bml_import_from_dense(2, 2, 0, n, M, H.ctypes.data_as(C.c_void_p), 0.05, 0)
    h = O.ref_ellpack_arrays(A)
    out = {"value": h[0], "index": h[1], "nnz": h[2], "N": n, "M": M}
    O.ref_free(A)
    np.savez_compressed(os.path.join(HERE, "hamiltonian600.npz"), **out)
    print("hamiltonian600.npz written")


if __name__ == "__main__":
    if sys.argv[1:] == ["hamiltonian"]:
        hamiltonian()
    else:
        main()
        hamiltonian()
