"""FP32-flux form: HLLC flux and limiter arithmetic in FP32, conserved-variable accumulation,
CFL reduction and floors in FP64 (the reference's FLOATFLUX option, cudaFluidStep.cu:118-122,
as a runtime switch).  Against the FP64 oracle the density must stay within 1e-5 relative L1."""
import numpy as np
import pytest

from gpuimogen_b200 import problems
from helpers import host, rel_l1, to_fluid

pytestmark = pytest.mark.gpu


# (392, 336, 6): z sweeps of a plane above 1 MB through the 8-column wide-block kernel;
# (1040, 520, 1): x rows above 1024 and y pencils above 512 cells through the chunked pipeline
# (160, 200, 2) and (96, 72, 4): rows and pencils of 65-127 and 129-255 cells, planes of a fixed
# 128- or 256-cell stride; (392, 336, 6): rows of 257-511 cells, a 512-cell stride
@pytest.mark.parametrize("shape,iters", [((48, 48, 48), 10), ((128, 96, 1), 20), ((512, 1, 1), 100),
                                         ((392, 336, 6), 3), ((1040, 520, 1), 3), ((160, 200, 2), 3),
                                         ((96, 72, 4), 5)])
def test_fp32_flux_close_to_fp64_oracle(cuda, ib, po, shape, iters):
    n = shape[0] * shape[1] * shape[2]
    q = problems.kelvin_helmholtz(shape, seed=5) if shape[1] > 1 else problems.sod(shape[0], 5 / 3.0)
    bc = "circular" if shape[1] > 1 else "const"
    fl = to_fluid(q, shape, bc=bc, gamma=5 / 3.0)
    geo = ib.Geometry(shape)
    tm = ib.TimeManager(cfl=0.4)
    num = ib.numerics(slope="mc", precision="fp32flux")
    ref = q.copy()
    sp = po.step_params(0.0, geo.h, 5 / 3.0, method=2, slope="mc")
    for it in range(iters):
        sp.dt = 0.4 * po.cfl_timestep(ref, shape, 5 / 3.0, geo.h, 2)
        po.fluid_step_3d(ref, shape, sp, [bc] * 6, 1, it)
        po.fluid_step_3d(ref, shape, sp, [bc] * 6, -1, it)
        ib.run_iteration([fl], geo, tm, 2, num)
    out = host(fl)
    err = rel_l1(out, ref, n)
    assert err[0] <= 1e-5, err          # density: the FP32-flux acceptance bound
    assert err[1] <= 1e-5, err          # total energy
    assert err[0] > 0                   # the FP32 path really ran
    assert np.all(np.isfinite(out[:, :n]))
