"""SW column unit with the reference's module interface (namgpu.physics.rrtm.phys_rrtm_sw_swrad.run);
phys-rrtm-grrad-sw loads it by name through its SWRAD_MODULE (phys_rrtm_grrad_sw.py:129)."""
from .driver import swrad_run as run  # noqa: F401
