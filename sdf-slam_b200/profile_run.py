"""Runs LM iterations of a synthetic workload through the public API and
prints the per-phase device times (CUDA events on the library's stream).

    python sdf-slam_b200/profile_run.py [workload] [iterations] [precision]

workload: room | floorplan | office (default floorplan). Each iteration is a
one-iteration solve call, so a profiler sees a fixed, repeating launch
sequence; the process loads no other CUDA library.
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _package():
    if "sdf_slam_b200" in sys.modules:
        return sys.modules["sdf_slam_b200"]
    spec = importlib.util.spec_from_file_location("sdf_slam_b200", os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sdf_slam_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    P = _package()
    import sdf_slam_b200.scenes as scenes
    workload = sys.argv[1] if len(sys.argv) > 1 else "floorplan"
    iterations = int(sys.argv[2]) if len(sys.argv) > 2 else 3
    precision = sys.argv[3] if len(sys.argv) > 3 else "fp64"
    sc = scenes.WORKLOADS[workload]()
    prob = P.Problem.from_scene(sc)
    specs = prob.specs(min_corner=sc.min_corner, max_corner=sc.max_corner)
    gpu = P.Problem.from_specs(specs)
    opts = P.SolverOptions(max_iterations=1, step_tolerance=0.0, precision=precision)
    for it in range(iterations):
        r = P.solve(gpu, opts)
        prof = gpu.last_profile()
        print(f"iteration {it}: cost {r.final_cost:.9e} " +
              " ".join(f"{k}={v * 1e3:.3f}ms" if isinstance(v, float) and k != "factor_flops" else f"{k}={v}"
                       for k, v in prof.items()))


if __name__ == "__main__":
    main()
