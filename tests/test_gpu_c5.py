"""The waveguide-variant study in small: material variants of one mesh on the
device (the 1/eps override equals a build with those materials, to the bit),
the TE10 incident-field source and per-step port amplitudes, and the
tensor-core stage kernel's port series against the FP32 kernel's."""
import ctypes as C

import numpy as np
import pytest

from rapidfem_b200 import _native as nat
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200 import td as T
from rapidfem_b200 import workloads as W

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_waveguide_variants_port_series():
    a, L = 22.86e-3, 60e-3
    wl = W.waveguide_post(6.0, order=2, cells=(8, 4, 16))
    op = wl.build()
    cen = wl.mesh.nodes[wl.mesh.tets].mean(axis=1)
    post = np.hypot(cen[:, 0] - a / 2, cen[:, 2] - L / 2) < 1.5e-3
    assert post.any()
    prof_in = op.rect_port_profiles(0, [0, 0, 1.0], (1, 0))
    prof_out = op.rect_port_profiles(1, [0, 0, -1.0], (1, 0))
    src = op.port_source(0, prof_in)
    funcs = [op.port_modal_weights(1, prof_out, "E"), op.port_modal_weights(0, prof_in, "E")]
    ctx = G.GpuContext(0)
    vac = G.GpuOperator(ctx, op, inv_eps=np.ones(3 * op.n_elem))
    rho = C.c_double()
    nat.check(nat.lib.dgtd_power_rho(vac.handle, 30, C.byref(rho)))
    dt = 0.5 * 2.8 / rho.value
    c = 299792458.0
    tau = 2.0 * np.sqrt(np.log(2.0)) / (np.pi * 4e9) * c
    steps = 300
    g = T.GaussianPulse(3 * tau, tau, 10e9 / c)(np.arange(steps) * dt).astype(np.float32)
    for eps in (2.0, 10.0):
        ie = np.repeat(np.where(post, 1.0 / eps, 1.0), 3)
        got = {}
        for eng in (nat.ENGINE_FP32, nat.ENGINE_TF32X3):
            gop = G.GpuOperator(ctx, op, inv_eps=ie)
            gop.set_engine(eng)
            got[eng], _ = gop.transient_functionals(np.zeros(op.n_dof), dt, steps, 1, drive=("vector", src), g=g,
                                                    functionals=funcs)
        built = O.MaxwellOperator(wl.mesh, 2, 1.0, face_port=wl.face_port,
                                  materials=O.isotropic_materials(np.where(post, eps, 1.0)))
        ref_op = G.GpuOperator(ctx, built)
        ref_op.set_engine(nat.ENGINE_FP32)
        ref, _ = ref_op.transient_functionals(np.zeros(op.n_dof), dt, steps, 1, drive=("vector", src), g=g,
                                              functionals=funcs)
        assert np.array_equal(got[nat.ENGINE_FP32], ref)
        assert rel_l2(got[nat.ENGINE_TF32X3][:, 0], ref[:, 0]) < 1e-4
        assert rel_l2(got[nat.ENGINE_TF32X3][:, 1], ref[:, 1]) < 1e-4
        assert np.max(np.abs(ref[:, 1])) > 0 and np.all(np.isfinite(ref))
