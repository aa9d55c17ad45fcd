"""LW column unit with the reference's module interface (namgpu.physics.rrtm.phys_rrtm_lw_lwrad.run);
phys-rrtm-grrad-lw loads it by name through its LWRAD_MODULE (phys_rrtm_grrad_lw.py:79)."""
from .driver import lwrad_run as run  # noqa: F401
