"""Backend markers: the B200 engine as two more members of the reference's backend family.

The reference selects its executor by dispatch on singleton marker types
(src/backends.jl:14-44: CPUBackend, GPUBackend, CPU_GCBackend, GPU_GCBackend).
``B200Backend`` is the Cartesian/radial executor (the GPUBackend's slot) and
``B200_GCBackend`` the Milne (τ, r) executor (the GPU_GCBackend's slot).
"""


class AbstractBackend:
    """Supertype of every simulation backend (backends.jl:14)."""


class B200Backend(AbstractBackend):
    """Fused sm_100a kernels, Cartesian or radial coordinates."""

    def __repr__(self):
        return "B200Backend()"


class B200_GCBackend(AbstractBackend):
    """Fused sm_100a kernels, Milne (τ, r) general coordinates."""

    def __repr__(self):
        return "B200_GCBackend()"
