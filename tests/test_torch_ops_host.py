"""The operator registration of thruster_cx_code_b200.torch_ops, without a GPU: the three
operators exist in torch.ops.pbemcs with the reference functions' argument names, declare
the tensors they mutate, and have no CPU kernel (CPU tensors raise, never fall back)."""
import pytest

torch = pytest.importorskip("torch")


def _schema(op):
    import thruster_cx_code_b200.torch_ops  # noqa: F401
    return getattr(torch.ops.pbemcs, op).default._schema


def test_operators_registered_with_reference_arguments():
    s = _schema("accumulate_rho")
    assert [a.name for a in s.arguments] == ["x", "y", "rho", "num_p", "dx", "dy", "nx", "ny", "charge_density"]
    s = _schema("push_particles_boris")
    assert [a.name for a in s.arguments][:10] == ["x", "y", "vx", "vy", "vz", "Ex", "Ey", "Bx", "By", "Bz"]
    s = _schema("thermal_conduction")
    assert [a.name for a in s.arguments] == ["T", "T_new", "mask", "nx", "ny", "Fo_x", "Fo_y"]


def test_mutated_arguments_declared():
    def mutated(op):
        return {a.name for a in _schema(op).arguments if a.alias_info is not None and a.alias_info.is_write}
    assert mutated("accumulate_rho") == {"rho"}
    assert mutated("push_particles_boris") == {"x", "y", "vx", "vy", "vz"}
    assert mutated("thermal_conduction") == {"T_new"}


def test_cpu_tensors_have_no_kernel():
    import thruster_cx_code_b200.torch_ops  # noqa: F401
    x = torch.zeros(4)
    rho = torch.zeros((4, 4))
    with pytest.raises(Exception):
        torch.ops.pbemcs.accumulate_rho(x, x, rho, 4, 0.1, 0.1, 4, 4, 1.0)
    assert rho.abs().sum().item() == 0.0
