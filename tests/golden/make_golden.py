"""Generates the small golden fixtures in tests/golden/ from the FP64 oracle.

The reference (MATLAB) cannot run here, so these fixtures freeze the oracle's
outputs on small seeded problems: the system matrices of both geometries and
SIRT/ART iterates.  tests/test_oracle.py checks that the oracle still
reproduces them; the GPU tests check libairt against them.

Run:  python tests/golden/make_golden.py         (all fixtures)
      python tests/golden/make_golden.py widened (widened_N16.npz only)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import airt_oracle as O  # noqa: E402


def problem(N=16, theta=None, eta=0.01, seed=3):
    theta = np.arange(0.0, 180.0, 6.0) if theta is None else theta
    A = O.paralleltomo_matrix(N, theta)
    x = O.shepplogan(N)
    bex = A @ x
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(bex.size)
    e = eta * np.linalg.norm(bex) * e / np.linalg.norm(e)
    return A, x, bex + e, float(np.linalg.norm(e)), theta


def main():
    A, x, b, enorm, theta = problem()
    np.savez_compressed(os.path.join(HERE, "paralleltomo_N16_30ang.npz"),
                        indptr=A.indptr, indices=A.indices, data=A.data, shape=A.shape,
                        theta=theta, x=x, b=b, enorm=enorm)
    F = O.fanlineartomo_matrix(12, np.arange(0.0, 360.0, 12.0), 17)
    np.savez_compressed(os.path.join(HERE, "fanlineartomo_N12_30ang.npz"),
                        indptr=F.indptr, indices=F.indices, data=F.data, shape=F.shape)
    out = {}
    for meth in ("landweber", "cimmino", "cav", "drop", "sart"):
        X, info, _ = O.sirt(meth, A, b, [5, 20], options={"lbound": 0.0, "ubound": 1.0})
        out[meth + "_X"] = X
        out[meth + "_rho"] = info["rho"]
    X, info, _ = O.sirt("cimmino", A, b, [200], options={
        "stoprule": {"type": "DP", "taudelta": 1.02 * enorm}, "rho": out["cimmino_rho"]})
    out["cimmino_dp_X"] = X
    out["cimmino_dp_finaliter"] = info["finaliter"]
    Xk, _ = O.art("kaczmarz", A, b, [2, 5], options={"lbound": 0.0})
    out["kaczmarz_X"] = Xk
    Xs, _ = O.art("symkaczmarz", A, b, [4], options={})
    out["symkaczmarz_X"] = Xs
    np.savez_compressed(os.path.join(HERE, "solvers_N16_30ang.npz"), **out)
    widened(A, b, theta)
    print("written", sorted(os.listdir(HERE)))


def f32(A):
    """A with FP32-rounded values, as libairt stores it (CART's flagging
    decisions and fbp are compared on this matrix)."""
    R = A.tocsc(copy=True)
    R.data = R.data.astype(np.float32).astype(np.float64)
    return R


def widened(A, b, theta):
    """widened_N16.npz: seismictomo (N=12, 6 sources, 10 receivers) and
    sphericaltomo (N=10, 12 centres, 8 circles) matrices, CART columnaction
    iterates with flagging, and fbp with two filters, on the paralleltomo
    N=16 problem with FP32-rounded values."""
    S = O.seismictomo_matrix(12, 6, 10)
    Q = O.sphericaltomo_matrix(10, np.arange(0.0, 360.0, 30.0), 8)
    R = f32(A)
    opts = {"lbound": 0.0, "Kbegin": 2, "Nunflag": 2, "THR": 1e-2, "seed": 5}
    Xc, ic = O.cart("columnaction", R, b, [2, 6], None, opts)
    out = dict(seis_indptr=S.indptr, seis_indices=S.indices, seis_data=S.data, seis_shape=S.shape,
               sph_indptr=Q.indptr, sph_indices=Q.indices, sph_data=Q.data, sph_shape=Q.shape,
               cart_X=Xc, cart_finaliter=ic["finaliter"],
               fbp_ramlak=O.fbp(R, b, theta, "ram-lak"), fbp_hamming=O.fbp(R, b, theta, "hamming"))
    np.savez_compressed(os.path.join(HERE, "widened_N16.npz"), **out)


if __name__ == "__main__":
    if sys.argv[1:] == ["widened"]:
        A, x, b, enorm, theta = problem()
        widened(A, b, theta)
    else:
        main()
