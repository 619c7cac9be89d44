"""Generates tests/golden/motion_golden.npz from the reference's own Motion.py.

Run in a container where the reference tree is present:
    python tests/golden/make_motion_golden.py /path/to/reference

python/feelmri/Motion.py imports feelmri.MPIUtilities (mpi4py) and the
compiled feelmri.POD; neither is available, so two stand-ins are injected:
MPI_print does nothing and MPI_rank is 0, and tensordot_modes_weights is the
float32 contraction numpy.einsum("pcm,m->pc").  Everything else -- the
periodic fold with NumPy's scalar promotion, the batched PPoly evaluation, the
float32 cast of the weights, the velocity scaling and the sums -- is the
reference's code.  For every case the file stores the state needed to rebuild
the callable (PPoly coefficients and breakpoints, modes, period and timeshift
with their NumPy types), the times passed to it, the float32 weights it
computed and its float32 output.
"""
from __future__ import annotations

import sys
import types
from pathlib import Path

import numpy as np


def load_reference_motion(ref_root: Path):
    pkg = types.ModuleType("feelmri")
    pkg.__path__ = [str(ref_root / "python" / "feelmri")]
    mpi = types.ModuleType("feelmri.MPIUtilities")
    mpi.MPI_print = lambda *a, **k: None
    mpi.MPI_rank = 0
    pod = types.ModuleType("feelmri.POD")
    pod.tensordot_modes_weights = lambda modes, w: np.einsum("pcm,m->pc", modes, w).astype(modes.dtype)
    sys.modules.update({"feelmri": pkg, "feelmri.MPIUtilities": mpi, "feelmri.POD": pod})
    import importlib.util
    spec = importlib.util.spec_from_file_location("feelmri.Motion", ref_root / "python" / "feelmri" / "Motion.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def kind_name(v) -> str:
    if v is None:
        return "none"
    if isinstance(v, np.float32):
        return "f32"
    if isinstance(v, np.float64):
        return "f64"
    return "py"


def main(ref_root: str) -> None:
    M = load_reference_motion(Path(ref_root))
    rng = np.random.default_rng(7)
    out = {}
    n_nodes, n_t = 37, 12

    def snapshots(n_modes):
        base = rng.normal(size=(n_nodes, 3, n_modes))
        tw = np.sin(np.linspace(0, 2 * np.pi, n_t)[:, None] * (1 + np.arange(n_modes))[None, :])
        return np.einsum("pcm,tm->pct", base, tw) + 1e-3 * rng.normal(size=(n_nodes, 3, n_t))

    cases = []
    # periodic POD, float32 knot times (float32 period), several timeshift types
    times32 = np.linspace(0, 900.0, n_t).astype(np.float32)
    times64 = np.linspace(0, 900.0, n_t)
    for name, cls, times, periodic, ts in [
        ("pod_p32_tspy", M.POD, times32, True, 125.5),
        ("pod_p32_ts32", M.POD, times32, True, np.float32(333.25)),
        ("pod_p32_ts64", M.POD, times32, True, np.float64(612.125)),
        ("pod_p64_tspy", M.POD, times64, True, 47.0),
        ("pod_nonper", M.POD, times64, False, 0.0),
        ("podvel_p32", M.PODVelocity, times32, True, 250.0),
        ("podvel_p64_ts32", M.PODVelocity, times64, True, np.float32(80.5)),
    ]:
        obj = cls(times=times, data=snapshots(3), n_modes=3, is_periodic=periodic, interpolation_method="Pchip")
        obj.update_timeshift(ts)
        cases.append((name, obj))
    resp = M.RespiratoryMotion(times=np.linspace(0, 3000.0, 50), data=0.008 * (1 - np.cos(np.linspace(0, np.pi, 50)) ** 4),
                               is_periodic=True, direction=np.array([0, 1, 0]), interpolation_method="Pchip")
    cases.append(("resp", resp))
    inner = M.POD(times=times32, data=snapshots(2), n_modes=2, is_periodic=True, interpolation_method="Pchip")
    psum = resp + inner
    psum.update_timeshift(np.float64(1500.0))
    cases.append(("sum_resp_pod", psum))

    # call times: float32 running times as the Bloch sweep passes them, knot
    # times, values beyond the period and negative values
    t_calls = np.concatenate([
        np.add.accumulate(np.full(40, 0.37, np.float32), dtype=np.float32).astype(np.float64),
        times32.astype(np.float64), [0.0, 899.99, 900.0, 1234.5, 4321.0, -10.0, -899.5],
    ])

    for name, obj in cases:
        outs = []
        weights = []
        for t in t_calls:
            y = np.asarray(obj(float(t)), dtype=np.float32)
            outs.append(np.broadcast_to(y, (n_nodes, 3)) if y.shape != (n_nodes, 3) else y)
            w = getattr(obj, "_weights", None)
            weights.append(np.array(w, dtype=np.float32) if w is not None else np.zeros(0, np.float32))
        out[f"{name}/t"] = t_calls
        out[f"{name}/out"] = np.stack(outs).astype(np.float32)
        out[f"{name}/weights"] = np.stack(weights)
        terms = [obj.pod1, obj.pod2] if hasattr(obj, "pod1") else [obj]
        out[f"{name}/n_terms"] = np.array(len(terms))
        for k, term in enumerate(terms):
            p = f"{name}/term{k}/"
            if hasattr(term, "_pp_batch"):
                out[p + "kind"] = np.array("PODVelocity" if type(term).__name__ == "PODVelocity" else "POD")
                out[p + "c"] = term._pp_batch.c
                out[p + "x"] = term._pp_batch.x
                out[p + "extrapolate"] = np.array(bool(term._pp_batch.extrapolate))
                out[p + "modes"] = term._modes
            else:
                out[p + "kind"] = np.array("RespiratoryMotion")
                out[p + "c"] = term.interpolator.c
                out[p + "x"] = term.interpolator.x
                out[p + "extrapolate"] = np.array(bool(term.interpolator.extrapolate))
                out[p + "direction"] = term.direction
            out[p + "timeshift"] = np.array(float(term.timeshift))
            out[p + "timeshift_kind"] = np.array(kind_name(term.timeshift))
            out[p + "period"] = np.array(float(term._period) if term._period is not None else 0.0)
            out[p + "period_kind"] = np.array(kind_name(term._period))
    out["cases"] = np.array([n for n, _ in cases])
    dest = Path(__file__).resolve().parent / "motion_golden.npz"
    np.savez_compressed(dest, **out)
    print(f"wrote {dest} ({dest.stat().st_size} bytes, {len(cases)} cases)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_motion_golden.py <path to the reference checkout>")
    main(sys.argv[1])
