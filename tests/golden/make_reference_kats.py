"""Writes reference_kats.json: the known-answer values the reference's own unit tests assert for the hot path.

The reference cannot be built in this environment (Eigen 3.2 / TBB / GL / SCons IEBuild are absent), so these
values are transcribed from the assertions in its test sources, each with its file:line, not computed by running
it.  tests/test_oracle_reference.py checks the oracle against them; the GPU parity tests then check the CUDA path
against the oracle.
"""
import json
import os

KATS = {
    "shape_function": {
        "source": "src/tests/TestShapeFunction.cpp:20-42,128-131",
        "w_at_support_radius": 0.0, "dw_at_support_radius": 0.0, "partition_of_unity_tol": 1e-6,
        "fd_derivative_tol": 1e-4, "fd_step": 0.001, "nodes_visited": 64, "sum_weights_tol": 1e-6,
        "grid_origin": [-1.7638, -2.85363, 2.25722], "particle": [0.15321, 2.29587345, -3.897576], "h": 0.314857,
    },
    "snow_clamp": {
        "source": "src/tests/TestSnowConstitutiveModel.cpp:30-36,67-76",
        "params": [1.0, 0.25, 10.0, 0.1, 0.2], "F_diag_in": [1.3, 0.8, 1.0], "F_diag_out": [1.2, 0.9, 1.0],
        "tol": 1e-4,
    },
    "deformation_gradient": {
        "source": "src/tests/TestGrid.cpp:216-278",
        "h": 0.2, "dt": 0.01, "steps": 7, "F00": "1 + 0.01 i", "F11": "1 - 0.01 i", "F22": "1 + 0.005 i",
        "tol": 0.001,
    },
    "sim_init": {
        "source": "src/tests/TestSimClass.cpp:45-118",
        "h": 0.1, "n_bodies": 2, "body_sizes": [4096, 4096], "n_ballistic": 4096, "n_variables_dummy_model": 5,
    },
    "sim_advance": {
        "source": "src/tests/TestSimClass.cpp:120-190",
        "h": 0.1, "dt": 0.01, "steps": 3, "gravity": [0.0, 1.0, 0.0], "mean_vy": 0.03, "vy_tol": 1e-5,
        "vxz_tol": 1e-6, "params": [1.4e5, 0.2, 0.0, 1e5, 1e5], "max_iters": 10, "tol": 0.0,
    },
    "cr_dense": {
        "source": "src/tests/TestConjugateResiduals.cpp:43-102",
        "n": 6, "residual_tol": 1e-3, "orthogonality_tol": 1e-4,
    },
    "implicit_update": {
        "source": "src/tests/TestGrid.cpp:456-708",
        "h": 0.5, "dt": 0.002, "iters": 40, "normal_velocity_tol": 1e-5, "equation_max_norm_tol": 1e-6,
    },
    "forces": {"source": "src/tests/TestGrid.cpp:281-396", "equilibrium_tol": 1e-4, "force_fd_rel": 0.01,
               "differential_fd_rel": 0.025},
    "dfidxi": {"source": "src/tests/TestGrid.cpp:806-852", "tol": 1e-8},
}

if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(out, "w") as f:
        json.dump(KATS, f, indent=1, sort_keys=True)
    print("wrote", out)
