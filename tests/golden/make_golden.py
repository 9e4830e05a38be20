"""Generate the golden fixtures in this folder from the reference itself.

    python tests/golden/make_golden.py REFERENCE_TREE

Needs the reference tree (its path is the one argument) and the checker libraries
built by oracle/Makefile (oracle/_ref/libref_cpu.so is the reference's own
src/pfaffian_cpu.cpp).  Outputs, all seeded and reproducible:

  cpu_f64.npz      inputs and Pf values from the reference's pfaffian_cpu
                   (src/pfaffian_cpu.cpp), as shipped: n = 2..32 (A = G - G^T,
                   rng 123, as test/pfaffian_test.py:67-78), 64 matrices of the
                   32x32 benchmark batch (A = (G - G^T)/2, rng 0), and n = 64, 128
                   with entries N(0, 1/n).
  cpu_large.npz    Pf from pfaffian_cpu for n = 256, 512, 1024 (entries
                   N(0, 1/n), seeds stored; matrices regenerated by the test).
  py_c128.npz      inputs and values of the reference's NumPy path
                   (pfcuda/pfaffian_py.py) on complex128 matrices.
Ragged collections are stored flattened and concatenated, with the orders in
`*_n` / `n`; tests/golden_io.py splits them again.

  known.npz        the reference's exact-answer construction
                   (test/pfaffian_test.py:80-109): B A B^T and its Pf.
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def load_pfaffian_py(ref):
    spec = importlib.util.spec_from_file_location("ref_pfaffian_py", os.path.join(ref, "pfcuda", "pfaffian_py.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.pfaffian_py


def main(ref):
    if O.ref_cpu() is None:
        raise SystemExit("build oracle/_ref first: make -C oracle")
    pf_py = load_pfaffian_py(ref)

    # --- reference CPU, small sizes
    rng = np.random.default_rng(123)
    sizes_A, sizes_n = [], []
    for n in range(2, 33, 2):
        for _ in range(4):
            G = rng.normal(size=(n, n))
            sizes_A.append(G - G.T)
            sizes_n.append(n)
    sizes_pf = np.array([O.ref_cpu_pfaffian(a) for a in sizes_A])
    bench = O.config_small(seed=0)[:64]
    bench_pf = O.ref_cpu_pfaffian(bench)
    rng = np.random.default_rng(7)
    mid = {}
    for n in (64, 128):
        A = O.skew_normal(rng, 3, n, scale=1.0 / np.sqrt(n))
        mid[n] = (A, O.ref_cpu_pfaffian(A))
    np.savez_compressed(
        os.path.join(HERE, "cpu_f64.npz"),
        sizes_A=np.concatenate([a.ravel() for a in sizes_A]), sizes_n=np.array(sizes_n), sizes_pf=sizes_pf,
        bench_A=bench, bench_pf=bench_pf,
        mid64_A=mid[64][0], mid64_pf=mid[64][1], mid128_A=mid[128][0], mid128_pf=mid[128][1])

    # --- reference CPU, large sizes (seeds only)
    seeds, ns, pfs = [], [], []
    for n, seed in ((256, 11), (512, 12), (1024, 13)):
        A = O.config_large(n, seed=seed)[0]
        seeds.append(seed)
        ns.append(n)
        pfs.append(O.ref_cpu_pfaffian(A))
    np.savez_compressed(os.path.join(HERE, "cpu_large.npz"), seeds=np.array(seeds), n=np.array(ns),
                        pf=np.array(pfs))

    # --- reference NumPy path on complex128
    rng = np.random.default_rng(5)
    cA, cn, cpf = [], [], []
    for n in (6, 8, 16, 32, 40):
        for _ in range(3):
            A = O.skew_normal(rng, 1, n, complex_=True)[0]
            cA.append(A.ravel())
            cn.append(n)
            cpf.append(complex(pf_py(A.copy())))
    np.savez_compressed(os.path.join(HERE, "py_c128.npz"), A=np.concatenate(cA), n=np.array(cn),
                        pf=np.array(cpf))

    # --- exact-answer construction
    rng = np.random.default_rng(0)
    kA, kn, kpf = [], [], []
    for n in list(range(2, 33, 2)) + [40, 64]:
        for _ in range(2):
            A, pf = O.tridiag_known(rng, n)
            kA.append(A.ravel())
            kn.append(n)
            kpf.append(pf)
    np.savez_compressed(os.path.join(HERE, "known.npz"), A=np.concatenate(kA), n=np.array(kn),
                        pf=np.array(kpf))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_TREE")
    main(sys.argv[1])
