"""The tcgen05 instruction and shared-memory descriptor encoders
(csrc/tc_ptx.cuh), decoded field by field on the host against the PTX ISA
layouts for every shape and operand address the kernels issue
(tests/descriptors_check.cu; no GPU needed)."""
from harness import run_host_check


def test_descriptor_fields(sb):
    assert run_host_check("descriptors_check").strip().endswith("descriptors ok")
