"""grrad's aerosol unit with the reference's module interface
(namgpu.physics.rrtm.phys_rrtm_grrad_aerosols.run(ctx, lsswr=, lslwr=)): the climatological aerosol optics
written to ctx.tables["rrtm_faersw"] / ["rrtm_faerlw"], where the LW and SW units read them."""
from .driver import grrad_aerosols_run as run  # noqa: F401
