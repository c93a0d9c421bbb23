"""The adjoint's local derivatives, checked in f64 on the host (no GPU).

The reverse stages of ns_world_vjp rest on a dual-number restatement of each forward function
(warm start, push, relax, prepare, the body stages, recycled separations, the manifolds of
every shape pair and restitution). ns_adjoint_selfcheck evaluates that restatement in f64 at seeded random inputs and
compares its vector-Jacobian product, direction by direction, with central differences of the
same function; and it compares the hand-derived reverse sweeps the solver stages run on the
GPU (warm start, push, relax, integrate positions and velocities, the relative normal velocity
restitution samples) with the dual-number products, which they must reproduce to rounding.
"""
import pytest

from natsel_b200.world import ADJOINT_CHECKS, adjoint_selfcheck

K_FACE_A, K_FACE_B, K_EDGE = 2, 3, 4


@pytest.mark.parametrize("which", range(9), ids=ADJOINT_CHECKS[:9])
def test_local_vjp_matches_central_differences(which):
    for seed in range(6):
        worst, _ = adjoint_selfcheck(which, seed)
        assert 0.0 <= worst < 1e-6, (ADJOINT_CHECKS[which], seed, worst)


@pytest.mark.parametrize("which", [9, 10, 11], ids=ADJOINT_CHECKS[9:12])
def test_box_manifold_vjp_matches_central_differences(which):
    kinds = set()
    for seed in range(16):
        worst, kind = adjoint_selfcheck(which, seed)
        assert 0.0 <= worst < 1e-6, (ADJOINT_CHECKS[which], seed, worst, kind)
        kinds.add(kind)
    if which == 9:
        assert K_FACE_A in kinds
    if which == 11:
        assert K_EDGE in kinds, kinds  # the edge-pair manifold is exercised


@pytest.mark.parametrize("which", range(12, 17), ids=ADJOINT_CHECKS[12:17])
def test_reverse_sweeps_match_dual_numbers(which):
    for seed in range(16):
        worst, _ = adjoint_selfcheck(which, seed)
        assert 0.0 <= worst < 1e-12, (ADJOINT_CHECKS[which], seed, worst)


def test_restitution_vjp_matches_central_differences():
    """The restitution update (contact_solver.rs:1135 apply_restitution_body) on one to four
    points; even seeds arm every point's bounce (relative velocity below the threshold)."""
    for seed in range(24):
        worst, _ = adjoint_selfcheck(17, seed)
        assert 0.0 <= worst < 1e-6, (seed, worst)


def test_relative_velocity_reverse_sweep_matches_dual_numbers():
    for seed in range(16):
        worst, _ = adjoint_selfcheck(18, seed)
        assert 0.0 <= worst < 1e-12, (seed, worst)


@pytest.mark.parametrize("which", range(19, 24), ids=ADJOINT_CHECKS[19:24])
def test_round_manifold_vjp_matches_central_differences(which):
    """Sphere and capsule pairs: the dual-number manifold replay against central differences at
    random touching poses, with the two-point capsule branch and every box-sphere and box-capsule
    path exercised."""
    seen = set()
    for seed in range(16):
        worst, kind = adjoint_selfcheck(which, seed)
        assert 0.0 <= worst < 1e-6, (ADJOINT_CHECKS[which], seed, worst, kind)
        seen.add(int(kind))
    if which == 21:
        assert seen == {1, 2}, seen  # one- and two-point manifolds
    if which == 22:
        assert seen == {2, 4}, seen  # distance path and the centre inside the box
    if which == 23:
        assert seen == {2, 3, 4, 5}, seen


@pytest.mark.parametrize("which", [24, 25, 26], ids=["joint_solve", "joint_warm_start", "joint_prepare"])
def test_joint_vjp_matches_central_differences(which):
    """Revolute joints (revolute_joint.rs:183-553): the solve with and without bias, with the
    spring, the motor (clamped and not) and the limits in turn; the warm start; the prepare."""
    for seed in range(12):
        worst, _ = adjoint_selfcheck(which, seed)
        assert 0.0 <= worst < 1e-6, (which, seed, worst)
