"""CPU restatement of the reference's Ceres backend, for the Ceres-parity
comparison harness.

TEST INFRASTRUCTURE ONLY: imported by tests/. The product library never loads
it.

What the reference's `SolveCeres` (src/solvers/ceres_solver.cpp:128-224) hands
to Ceres is restated exactly:
* one point residual per point spec whose point, at the poses of the solve's
  start, lies in the grid and whose cell's four nodes are all active: the
  frozen-cell residual `EvalPointResidualFrozenCell`
  (src/problem/residual_math.hpp:113-147), times the spec's sqrt weight,
  under a Huber loss when the problem has a Huber delta (:162-176);
* one Eikonal residual per Eikonal spec whose three nodes are active
  (`EikonalCost`, :64-93, :178-187);
* one odometry residual per odometry spec (`OdomCost`, :95-124, :189-193);
* frame 0's pose held constant (:195-197);
* the solution copied back with wrapped angles, and the result's costs taken
  from the problem's own Cost() (:200-223).

Ceres itself is a third-party library absent from this image
(`find_package(Ceres)`, CMakeLists.txt:17, version unpinned), so its solver
is restated from its published Levenberg-Marquardt trust-region algorithm
with the options SolveCeres sets (:199-208) and Ceres's defaults otherwise:
* Jacobi scaling of the columns by 1 / (1 + column norm);
* an LM diagonal of the squared scaled column norms, clamped to
  [1e-6, 1e32], divided by the trust radius;
* an initial radius of 1 / max(lambda_init, 1e-12);
* a step that lowers the cost by more than 1e-3 of the model's prediction is
  taken, and the radius grows by 1 / max(1/3, 1 - (2 rho - 1)^3);
* otherwise the radius shrinks by a decrease factor that starts at 2 and
  doubles with each rejection;
* convergence tests: function tolerance 1e-6, gradient tolerance 1e-10, and
  parameter tolerance = step_tolerance.

The normal equations are solved by a sparse LU here, where Ceres uses sparse
Cholesky; a factorization that fails counts as an unsuccessful step, which
shrinks the radius. Parity with Ceres is unpinned, since Ceres cannot run here. The
restatement is pinned by the reference's own tests of the formulation: the
frozen-cell residual equals the regular one inside its cell
(tests/test_jacobians.cpp:78-102), and the CornerScan Ceres variant passes
the end-to-end recovery bounds (tests/test_e2e.cpp:155-166).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle as O


def frozen_cell_point(nx, ny, mn, mx, cell_w, cell_h, pose, p, delta, node_values):
    """EvalPointResidualFrozenCell (residual_math.hpp:113-147): the point
    residual with the cell (cell_w, cell_h) kept whatever the pose; returns
    (residual, d_nodes[4], node_ids[4], d_pose[3])."""
    dx = (mx[0] - mn[0]) / (nx - 1)
    dy = (mx[1] - mn[1]) / (ny - 1)
    c = math.cos(pose[2])
    s = math.sin(pose[2])
    gx_ = c * p[0] - s * p[1] + pose[0]
    gy_ = s * p[0] + c * p[1] + pose[1]
    alpha = (gx_ - (mn[0] + cell_w * dx)) / dx
    beta = (gy_ - (mn[1] + cell_h * dy)) / dy
    w = np.array([(1.0 - alpha) * (1.0 - beta), alpha * (1.0 - beta), (1.0 - alpha) * beta, alpha * beta])
    v = np.asarray(node_values, dtype=np.float64)
    residual = -delta
    for i in range(4):
        residual += w[i] * v[i]
    ids = np.array([cell_h * nx + cell_w, cell_h * nx + cell_w + 1, (cell_h + 1) * nx + cell_w,
                    (cell_h + 1) * nx + cell_w + 1])
    gx = ((1.0 - beta) * (v[1] - v[0]) + beta * (v[3] - v[2])) / dx
    gy = ((1.0 - alpha) * (v[2] - v[0]) + alpha * (v[3] - v[1])) / dy
    dxt = -s * p[0] - c * p[1]
    dyt = c * p[0] - s * p[1]
    return residual, w, ids, np.array([gx, gy, gx * dxt + gy * dyt])


class CeresFormulation:
    """The residual blocks SolveCeres builds from a problem's specs at its
    current state (the cells frozen there), over the parameters: the active
    node values, then (x, y, theta) of frames 1..F-1."""

    def __init__(self, specs: "O.Specs"):
        self.s = specs
        nx, ny = specs.nx, specs.ny
        self.dx = (specs.max_corner[0] - specs.min_corner[0]) / (nx - 1)
        self.dy = (specs.max_corner[1] - specs.min_corner[1]) / (ny - 1)
        self.col = np.asarray(specs.node_to_active, dtype=np.int64)
        self.num_active = int(np.count_nonzero(self.col >= 0))
        self.num_frames = len(specs.poses)
        self.n = self.num_active + 3 * (self.num_frames - 1)
        poses = np.asarray(specs.poses, dtype=np.float64)
        # the point blocks: cells located at the solve's starting poses
        self.points = []
        for q in range(len(specs.pt_frame)):
            f = int(specs.pt_frame[q])
            loc = O.locate(nx, ny, specs.min_corner, specs.max_corner, specs.map_values,
                           self._apply(poses[f], specs.pt_xy[q]))
            if loc is None:
                continue
            w, h = loc["w"], loc["h"]
            ids = [h * nx + w, h * nx + w + 1, (h + 1) * nx + w, (h + 1) * nx + w + 1]
            if any(self.col[i] < 0 for i in ids):
                continue
            self.points.append((q, w, h, ids))
        self.eikonal = []
        for e in range(len(specs.eik_sqrtw)):
            w, h = int(specs.eik_wh[e][0]), int(specs.eik_wh[e][1])
            ids = [h * nx + w, h * nx + w + 1, (h + 1) * nx + w]
            if any(self.col[i] < 0 for i in ids):
                continue
            self.eikonal.append((e, ids))
        # Ceres holds only the parameter blocks some residual block uses: an
        # active node no block touches keeps its value
        used = np.zeros(self.n, dtype=bool)
        for q, _, _, ids in self.points:
            used[self.col[ids]] = True
            pc = self._pose_cols(int(specs.pt_frame[q]))
            if pc is not None:
                used[pc:pc + 3] = True
        for _, ids in self.eikonal:
            used[self.col[ids]] = True
        for o in range(len(specs.odom_sqrtw)):
            for f in specs.odom_ij[o]:
                pc = self._pose_cols(int(f))
                if pc is not None:
                    used[pc:pc + 3] = True
        self.used = np.nonzero(used)[0]

    @staticmethod
    def _apply(pose, p):
        c, s = math.cos(pose[2]), math.sin(pose[2])
        return (c * p[0] - s * p[1] + pose[0], s * p[0] + c * p[1] + pose[1])

    def pack(self, map_values, poses):
        x = np.zeros(self.n)
        act = np.nonzero(self.col >= 0)[0]
        x[self.col[act]] = np.asarray(map_values)[act]
        x[self.num_active:] = np.asarray(poses, dtype=np.float64)[1:].reshape(-1)
        return x

    def unpack(self, x):
        values = np.array(self.s.map_values, dtype=np.float64)
        act = np.nonzero(self.col >= 0)[0]
        values[act] = x[self.col[act]]
        poses = np.array(self.s.poses, dtype=np.float64)
        poses[1:] = x[self.num_active:].reshape(-1, 3)
        return values, poses

    def _pose_cols(self, f):
        return None if f == 0 else self.num_active + 3 * (f - 1)

    def evaluate(self, x, jacobian=True):
        """Ceres's cost 1/2 sum rho(|r|^2) and, when asked, the residuals and
        Jacobian after the loss's correction (for Huber, sqrt(rho') scales a
        block's residual and Jacobian)."""
        s = self.s
        values, poses = self.unpack(x)
        res, rows, cols, vals = [], [], [], []
        cost = 0.0
        delta = float(s.huber_delta)

        def block(r, entries):
            nonlocal cost
            sq = float(np.dot(r, r))
            scale = 1.0
            if delta > 0.0 and sq > delta * delta:
                cost += 0.5 * (2.0 * delta * math.sqrt(sq) - delta * delta)
                scale = math.sqrt(delta / math.sqrt(sq))
            else:
                cost += 0.5 * sq
            base = len(res)
            res.extend(scale * r)
            if jacobian:
                for k, c, v in entries:
                    rows.append(base + k)
                    cols.append(c)
                    vals.append(scale * v)

        for q, w, h, ids in self.points:
            f = int(s.pt_frame[q])
            r, dn, _, dp = frozen_cell_point(s.nx, s.ny, s.min_corner, s.max_corner, w, h, poses[f],
                                             s.pt_xy[q], float(s.pt_expected[q]), values[ids])
            sw = float(s.pt_sqrtw[q])
            ent = [(0, int(self.col[ids[k]]), sw * dn[k]) for k in range(4)]
            pc = self._pose_cols(f)
            if pc is not None:
                ent += [(0, pc + k, sw * dp[k]) for k in range(3)]
            block(np.array([sw * r]), ent)
        for e, ids in self.eikonal:
            nrm = s.eik_n[e]
            sw = float(s.eik_sqrtw[e])
            gx = (values[ids[1]] - values[ids[0]]) / self.dx
            gy = (values[ids[2]] - values[ids[0]]) / self.dy
            r = sw * (1.0 - (nrm[0] * gx + nrm[1] * gy))
            ent = [(0, int(self.col[ids[0]]), sw * (nrm[0] / self.dx + nrm[1] / self.dy)),
                   (0, int(self.col[ids[1]]), -sw * nrm[0] / self.dx),
                   (0, int(self.col[ids[2]]), -sw * nrm[1] / self.dy)]
            block(np.array([r]), ent)
        for o in range(len(s.odom_sqrtw)):
            i, j = int(s.odom_ij[o][0]), int(s.odom_ij[o][1])
            r, ji, jj = O.eval_odom(poses[i], poses[j], s.odom_meas[o])
            sw = float(s.odom_sqrtw[o])
            ent = []
            for f, jac in ((i, ji), (j, jj)):
                pc = self._pose_cols(f)
                if pc is not None:
                    ent += [(a, pc + b, sw * jac[a, b]) for a in range(3) for b in range(3)]
            block(sw * np.asarray(r), ent)
        r = np.array(res)
        if not jacobian:
            return cost, r, None
        J = sp.csr_matrix((vals, (rows, cols)), shape=(len(res), self.n))
        return cost, r, J


def solve_ceres(specs: "O.Specs", max_iterations=100, step_tolerance=1e-6, lambda_init=1.0):
    """SolveCeres (ceres_solver.cpp:128-224) on a copy of `specs`' state with
    the Levenberg-Marquardt trust-region strategy restated above. Returns
    (map_values, poses with wrapped angles, result dict: converged,
    iterations as summary.iterations.size() counts them (the start
    included), initial_cost and final_cost from the problem's Cost(),
    ceres_cost)."""
    prob = CeresFormulation(specs)
    orc = O.OracleProblem.from_specs(specs)
    initial_cost = orc.cost()
    x = prob.pack(specs.map_values, specs.poses)
    radius = 1.0 / max(lambda_init, 1e-12)
    decrease = 2.0
    used = prob.used

    def jac(x_):
        c_, r_, J_ = prob.evaluate(x_)
        return c_, r_, J_[:, used]

    cost, r, J = jac(x)
    iterations = 1
    converged = False
    while iterations <= max_iterations:
        g = J.T @ r
        if np.max(np.abs(g), initial=0.0) <= 1e-10:
            converged = True
            break
        colnorm = np.sqrt(np.asarray(J.multiply(J).sum(axis=0)).ravel())
        scale = 1.0 / (1.0 + colnorm)
        Js = J @ sp.diags(scale)
        diag = np.clip(np.asarray(Js.multiply(Js).sum(axis=0)).ravel(), 1e-6, 1e32)
        A = (Js.T @ Js + sp.diags(diag / radius)).tocsc()
        iterations += 1
        try:
            dy = spla.splu(A).solve(-(Js.T @ r))
        except RuntimeError:  # a singular factorization: the step fails
            dy = None
        if dy is None or not np.all(np.isfinite(dy)):
            # a failed linear solve counts as an unsuccessful step
            radius /= decrease
            decrease *= 2.0
            if radius < 1e-32:
                break
            continue
        dx = np.zeros_like(x)
        dx[used] = scale * dy
        jd = Js @ dy
        model_change = -(float(r @ jd) + 0.5 * float(jd @ jd))
        if np.linalg.norm(dx) <= (np.linalg.norm(x[used]) + step_tolerance) * step_tolerance:
            converged = True
            break
        new_cost, _, _ = prob.evaluate(x + dx, jacobian=False)
        rho = (cost - new_cost) / model_change if model_change > 0.0 else -1.0
        if rho > 1e-3:
            x = x + dx
            done = abs(cost - new_cost) <= 1e-6 * cost
            cost, r, J = jac(x)
            radius = min(radius / max(1.0 / 3.0, 1.0 - (2.0 * rho - 1.0) ** 3), 1e16)
            decrease = 2.0
            if done:
                converged = True
                break
        else:
            radius /= decrease
            decrease *= 2.0
            if radius < 1e-32:
                break
    values, poses = prob.unpack(x)
    poses[:, 2] = np.arctan2(np.sin(poses[:, 2]), np.cos(poses[:, 2]))
    orc.set_state(values, poses)
    return values, poses, dict(converged=converged, iterations=iterations, initial_cost=initial_cost,
                               final_cost=orc.cost(), ceres_cost=cost,
                               residual_blocks=len(prob.points) + len(prob.eikonal) + len(specs.odom_sqrtw))


def observed_nodes(specs: "O.Specs"):
    """The nodes of the cells the point blocks froze: the part of the map the
    scans observe. Nodes outside it are held only by Eikonal terms, which fix
    differences between neighbours but not the level, so their values are
    not comparable between backends."""
    f = CeresFormulation(specs)
    return np.unique(np.concatenate([np.asarray(ids) for _, _, _, ids in f.points]))


def compare(lm_state, lm_result, ceres_state, ceres_result, nodes=None):
    """The comparison the reference makes between its backends: both runs'
    costs in the problem's own Cost(), and the largest pose and map
    differences between their final states (the map over `nodes`, all nodes
    when None)."""
    (lm_m, lm_p), (ce_m, ce_p) = lm_state, ceres_state
    dth = np.arctan2(np.sin(lm_p[:, 2] - ce_p[:, 2]), np.cos(lm_p[:, 2] - ce_p[:, 2]))
    sel = slice(None) if nodes is None else nodes
    return {"lm_final_cost": float(lm_result["final_cost"]), "ceres_final_cost": float(ceres_result["final_cost"]),
            "max_pose_diff_m": float(np.max(np.abs(lm_p[:, :2] - ce_p[:, :2]))),
            "max_angle_diff_rad": float(np.max(np.abs(dth))),
            "max_map_diff": float(np.max(np.abs(lm_m[sel] - ce_m[sel])))}
