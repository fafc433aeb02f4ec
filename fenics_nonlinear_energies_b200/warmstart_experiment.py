"""Learned vs plain Newton warm starts on hyperelastic load paths.

``python -m fenics_nonlinear_energies_b200.warmstart_experiment [--nx 80 --ny 4 --nz 4]
  [--train-paths 16 --test-paths 4 --steps 24] [--out results.json]``

1. Solve ``--train-paths`` load paths (right-face twist up to a random total
   angle in [2 pi, 6 pi], Young's modulus in [5, 20], seeded) with Newton
   from the plain previous-step start; every converged step solution is a
   training sample.
2. Train the nodal MLP (4 layers, width 256, BF16 weights, FP32 accumulate)
   on the step transitions with the project's kernels.
3. On ``--test-paths`` new random paths, solve every step twice: from the
   plain previous-step start and from the MLP prediction (accepted only if it
   reaches the same gradient tolerance and energy; otherwise the plain solve
   is used and both are charged).  Report total Newton iterations and time.
"""

from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from fenics_nonlinear_energies_b200 import meshes
from fenics_nonlinear_energies_b200.warmstart import BeamFeatures, mlp_predict, run_load_path, train_mlp, \
    training_pairs


def random_paths(n, seed):
    rng = np.random.default_rng(seed)
    return [(float(rng.uniform(2 * math.pi, 6 * math.pi)), float(rng.uniform(5.0, 20.0))) for _ in range(n)]


def run(nx=80, ny=4, nz=4, train_paths=16, test_paths=4, steps=24, epochs=150, seed=0, log=print):
    torch.cuda.set_device(0)
    t_all = time.perf_counter()
    feats = None
    F_all, T_all = [], []
    gen_its, gen_time, gen_steps, gen_fail = 0, 0.0, 0, 0
    fail_msgs = {}
    for i, (theta, E) in enumerate(random_paths(train_paths, seed)):
        params, _ = meshes.he_beam_problem(nx=nx, ny=ny, nz=nz, E=E)
        if feats is None:
            feats = BeamFeatures(params)
        t0 = time.perf_counter()
        recs, sols = run_load_path(params, theta, steps, E=E, record=True)
        gen_time += time.perf_counter() - t0
        gen_its += sum(r["plain_its"] for r in recs)
        gen_steps += len(recs)
        gen_fail += sum(not r["plain_converged"] for r in recs)
        for r in recs:
            if not r["plain_converged"]:
                fail_msgs[r["plain_message"]] = fail_msgs.get(r["plain_message"], 0) + 1
        F, T = training_pairs(feats, sols, theta, E)
        F_all.append(F)
        T_all.append(T)
        log(f"train path {i}: theta={theta:.3f} E={E:.2f} newton_its={sum(r['plain_its'] for r in recs)} "
            f"t={time.perf_counter() - t0:.1f}s")
    F, T = np.concatenate(F_all), np.concatenate(T_all)
    t0 = time.perf_counter()
    mlp, hist = train_mlp(F, T, epochs=epochs, seed=seed, log=log)
    torch.cuda.synchronize()
    train_time = time.perf_counter() - t0
    plain_its = learned_its = accepted = n_steps = 0
    plain_time = learned_time = 0.0
    per_path = []
    for j, (theta, E) in enumerate(random_paths(test_paths, seed + 1000)):
        params, _ = meshes.he_beam_problem(nx=nx, ny=ny, nz=nz, E=E)
        recs = run_load_path(params, theta, steps, E=E, predictor=lambda f: mlp_predict(mlp, f), features=feats)
        p = sum(r["plain_its"] for r in recs)
        q = sum(r["learned_its"] for r in recs)
        a = sum(r["accepted"] for r in recs)
        ps = sum(r["plain_s"] for r in recs)
        qs = sum(r["learned_s"] for r in recs)
        plain_its += p
        learned_its += q
        accepted += a
        n_steps += len(recs)
        plain_time += ps
        learned_time += qs
        per_path.append({"theta_total": theta, "E": E, "plain_its": p, "learned_its": q, "accepted_steps": a,
                         "plain_s": ps, "learned_s": qs,
                         "steps": len(recs), "plain_converged": all(r["plain_converged"] for r in recs)})
        log(f"test path {j}: plain {p} its {ps:.2f} s, learned {q} its {qs:.2f} s, accepted {a}/{len(recs)}")
    out = {
        "mesh": {"hexes": [nx, ny, nz], "tets": 6 * nx * ny * nz},
        "steps_per_path": steps, "train_paths": train_paths, "test_paths": test_paths,
        "training_samples": int(F.shape[0]), "training_step_solutions": int(F.shape[0] // len(feats.X)),
        "mlp": {"dims": [F.shape[1], 256, 256, 256, T.shape[1]], "dtype": "bf16 weights, fp32 accumulate",
                "epochs": epochs, "final_mse": hist[-1], "train_time_s": train_time},
        "generation": {"newton_its": gen_its, "steps": gen_steps, "failed_steps": gen_fail, "failure_messages": fail_msgs,
                       "time_s": gen_time},
        "test": {"plain_newton_its": plain_its, "learned_newton_its": learned_its, "accepted_steps": accepted,
                 "steps": n_steps, "reduction": 1.0 - learned_its / max(1, plain_its),
                 "plain_newton_s": plain_time, "learned_newton_s": learned_time,
                 "time_reduction": 1.0 - learned_time / max(1e-12, plain_time), "paths": per_path},
        "tolerance": "||g|| <= 1e-6 ||g_0|| per step", "total_time_s": time.perf_counter() - t_all,
    }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=80)
    ap.add_argument("--ny", type=int, default=4)
    ap.add_argument("--nz", type=int, default=4)
    ap.add_argument("--train-paths", type=int, default=16)
    ap.add_argument("--test-paths", type=int, default=4)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    res = run(a.nx, a.ny, a.nz, a.train_paths, a.test_paths, a.steps, a.epochs, a.seed)
    txt = json.dumps(res, indent=1)
    print(txt)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt)


if __name__ == "__main__":
    main()
