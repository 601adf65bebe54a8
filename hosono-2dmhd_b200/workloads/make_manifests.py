"""Draw the seeded inputs of the batched and served workloads and write them
as JSON manifests next to this script, so every consumer (GPU engine, CPU
oracle, tests) reads identical instances.

blast64_seed0.json -- 64 independent MHD blasts (explosion2d form) on
  [-0.5,0.5]^2, periodic, gamma=5/3, rho=1, p_out=0.1, radius 0.1,
  B = (10/sqrt(4 pi)) (cos theta, sin theta, 0); GP radius 2, ell/dx=6,
  CFL 0.8, t_end 0.02.  Per instance, in this order: N uniform on
  {128,192,256,384,512}; p_in/p_out log-uniform on [10, 1000]; theta uniform
  on [0, pi/2].  numpy.random.Generator(PCG64(0)).

served2000_seed1.json -- 2000 requests.  Per request, in this order: problem
  uniform on {OrszagTang, Sedov, blast}; N = round(exp(U[ln 64, ln 1024]));
  t_end factor uniform on [0.1, 1] (times the problem's default t_end: OT 0.5,
  Sedov 0.05, blast 0.02); GP radius uniform on {1, 2}; for a blast request
  p_in/p_out and theta as above; then a unit-mean exponential inter-arrival
  gap (scaled by 1/rate when the stream is replayed, the rate being 80% of
  the measured batched capacity).  numpy.random.Generator(PCG64(1)).
"""
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TEND = {"OrszagTang2d": 0.5, "sedov2d": 0.05, "explosion2d": 0.02}


def blast64(seed=0, n=64):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(n):
        N = int(rng.choice([128, 192, 256, 384, 512]))
        ratio = float(math.exp(rng.uniform(math.log(10.0), math.log(1000.0))))
        theta = float(rng.uniform(0.0, math.pi / 2))
        out.append(dict(id=k, problem="explosion2d", n=N, radius=2, ell=6.0, p_ratio=ratio, theta=theta,
                        tmax=0.02, cfl=0.8))
    return out


def served(seed=1, n=2000):
    rng = np.random.Generator(np.random.PCG64(seed))
    problems = ["OrszagTang2d", "sedov2d", "explosion2d"]
    out = []
    for k in range(n):
        prob = problems[int(rng.integers(0, 3))]
        N = int(round(math.exp(rng.uniform(math.log(64.0), math.log(1024.0)))))
        fac = float(rng.uniform(0.1, 1.0))
        R = int(rng.integers(1, 3))
        req = dict(id=k, problem=prob, n=N, radius=R, tmax=fac * DEFAULT_TEND[prob], tmax_factor=fac)
        if prob == "explosion2d":
            req["p_ratio"] = float(math.exp(rng.uniform(math.log(10.0), math.log(1000.0))))
            req["theta"] = float(rng.uniform(0.0, math.pi / 2))
        req["gap"] = float(rng.exponential(1.0))
        out.append(req)
    return out


def main():
    with open(os.path.join(HERE, "blast64_seed0.json"), "w") as f:
        json.dump(dict(seed=0, generator="numpy PCG64", instances=blast64()), f, indent=0)
    with open(os.path.join(HERE, "served2000_seed1.json"), "w") as f:
        json.dump(dict(seed=1, generator="numpy PCG64", requests=served()), f, indent=0)


if __name__ == "__main__":
    main()
