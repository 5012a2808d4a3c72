"""Generates the golden fixtures of the parity tests.

known_answers.json: the known-answer values of the reference's own unit and
end-to-end tests for this path, with the file:line they come from
(tests/test_grid_map.cpp, test_hallucination.cpp, test_pose.cpp,
test_jacobians.cpp, test_e2e.cpp, test_parallel_ldlt.cpp of RobinJehn/sdf-slam).
The reference cannot be built here (Eigen, Ceres, CHOLMOD, yaml-cpp, nanoflann
and googletest are absent), so its tests are restated: the values below are
the expectations those tests assert.

room_oracle.npz: the oracle's outputs on the seeded 10-pose room scene (the
40x40 / 0.25 m workload): specs built by the oracle's Problem constructor, the
first linearization (residuals, cells, -J^T r, step) and a 10-iteration LM
cost history. Regenerate with `python tests/golden/make_golden.py`.
"""
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _scenes():
    pkg_dir = os.path.join(ROOT, "sdf-slam_b200")
    spec = importlib.util.spec_from_file_location("sdfslam_scenes", os.path.join(pkg_dir, "scenes.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sdfslam_scenes"] = mod
    spec.loader.exec_module(mod)
    return mod


KNOWN = {
    "grid_map": {
        "source": "tests/test_grid_map.cpp:8-76",
        "nx": 3, "ny": 3, "min": [0.0, 0.0], "max": [2.0, 2.0], "values": "w + 10 h",
        "interpolation": {"p": [0.5, 0.25], "value": 0.5 * 0.75 * 1.0 + 0.5 * 0.25 * 10.0 + 0.5 * 0.25 * 11.0,
                          "tol": 1e-12},
        "gradient_fd": {"p": [0.7, 1.3], "eps": 1e-7, "tol": 1e-5},
        "grid_line": {"p": [1.0, 1.0], "w": 1, "h": 1, "alpha": 0.0, "beta": 0.0},
        "upper_boundary": {"p": [2.0, 2.0], "w": 1, "h": 1, "alpha": 1.0, "beta": 1.0},
        "outside": [[-0.1, 1.0], [1.0, 2.1]],
    },
    "hallucination": {
        "source": "tests/test_hallucination.cpp:8-54",
        "both": {"point": [4.0, 0.0], "per_point": 6, "step": 0.1, "count": 6,
                 "x": {"0": 3.9, "1": 4.1, "4": 3.7}, "expected": {"0": 0.1, "1": -0.1, "4": 0.3}},
        "one_direction": {"point": [0.0, 2.0], "per_point": 3, "step": 0.5, "count": 3},
        "zero_beam": {"point": [0.0, 0.0], "count": 0},
    },
    "pose": {
        "source": "tests/test_pose.cpp:8-32",
        "apply": {"pose": [1.0, 2.0, 1.5707963267948966], "p": [1.0, 0.0], "out": [1.0, 3.0]},
        "roundtrip": {"a": [0.3, -1.2, 0.7], "b": [-2.0, 4.5, -2.9]},
        "wrap": [[9.42477796076938, 3.141592653589793, "abs"], [-9.42477796076938, 3.141592653589793, "abs"],
                 [0.5, 0.5, "eq"], [6.533185307179586, 0.25, "eq"], [-6.533185307179586, -0.25, "eq"]],
    },
    "jacobians": {"source": "tests/test_jacobians.cpp:13-153", "eps": 1e-6, "tol": 1e-5,
                  "eikonal": {"node": [2, 1], "normal": [0.6, 0.8]},
                  "odom": {"pose_i": [0.5, -1.0, 0.9], "pose_j": [1.5, 0.25, 1.4], "meas": [0.9, 1.1, 0.45]}},
    "e2e": {"source": "tests/test_e2e.cpp:18-218", "max_iterations": 40,
            "bounds": {"cost_ratio": 0.05, "translation": 0.1, "rotation": 0.05, "surface_sdf": 0.1},
            "variants": ["lm", "relation", "trust_region", "huber_0.5", "active_region"]},
    "ldlt": {"source": "tests/test_parallel_ldlt.cpp:32-118", "sizes": "3000 + 500 * seed",
             "seeds": [11, 12, 13], "width": 57, "refactor": {"n": 4000, "width": 63, "diag_shift": 2.5},
             "singular": {"n": 600, "zero_at": 300}},
}


def main():
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(KNOWN, f, indent=1)
    import oracle as O
    S = _scenes()
    sc = S.room_scene(seed=0)

    class Opt:
        pass

    o = Opt()
    o.weights_scan = o.weights_hallucination = o.weights_eikonal = o.weights_odometry = o.weights_relation = 1.0
    o.hallucination_points = 4
    o.hallucination_step = 0.1
    o.hallucination_both = True
    o.normal_method = 2
    o.k_neighbors = 10
    o.normals_per_scan = False
    o.corner_threshold = 0.2
    o.huber_delta = 0.0
    o.smooth_gradient = True
    o.smooth_gradient_step = 0.0
    o.active_region = False
    o.active_margin = 2
    p = O.OracleProblem.build(sc.nx, sc.ny, sc.min_corner, sc.max_corner, sc.poses, sc.scans, sc.odometry, o)
    specs = p.specs(sc.nx, sc.ny, sc.min_corner, sc.max_corner)
    lin = p.linearize(1.0, False, 1, True)
    res = p.solve(max_iterations=10, num_threads=1)
    np.savez_compressed(
        os.path.join(HERE, "room_oracle.npz"),
        pt_frame=specs.pt_frame, pt_xy=specs.pt_xy, pt_expected=specs.pt_expected, pt_sqrtw=specs.pt_sqrtw,
        eik_wh=specs.eik_wh, eik_n=specs.eik_n, eik_sqrtw=specs.eik_sqrtw, odom_ij=specs.odom_ij,
        odom_meas=specs.odom_meas, odom_sqrtw=specs.odom_sqrtw, node_to_active=specs.node_to_active,
        poses=specs.poses, residuals=lin["residuals"], point_cell=lin["point_cell"], rhs=lin["rhs"],
        step=lin["step"], cost_history=np.array(res["cost_history"]))
    print("wrote", HERE)


if __name__ == "__main__":
    main()
