"""How a reverse march of the differentiable renderer's backward fares.

The backward needs each sample's transmittance T_i.  Reconstructing it from
the final transmittance by T_i = T_{i+1} / (1 - a_i) divides by 1 - a_i;
this measures, in FP32 on the CPU (oracle/mk_oracle.c,
mko_dvr_reverse_stats), how far that reconstruction drifts from the forward
values on the benchmark's workload (256^3 float phantom, 8 views of 256^2,
step 0.5 voxel, t_min 1e-4), and on the same workload with opaque LUT
entries, where it breaks (1 - a = 0).  The figures support the backward's
design in mk_dvr.cu (reverse march, reset at per-ray checkpoints, a
checkpoint re-march for opaque samples); they are reported, not a parity
check."""
import ctypes as C

import numpy as np

import oracle
from monkeygl_b200 import dvr
from monkeygl_b200.camera import view_camera
from monkeygl_b200.phantom import config_phantom, make_tf_control_points, make_tf_lut


def stats(vol, lut, views):
    L = oracle.cpu()
    L.mko_dvr_reverse_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    tot = np.zeros(5)
    for p in views:
        flat = dvr.params_flat(p)
        st = np.zeros(5)
        assert L.mko_dvr_reverse_stats(flat.ctypes.data, vol.ctypes.data, lut.ctypes.data, 0, st.ctypes.data) == 0
        tot[[0, 1, 2, 4]] += st[[0, 1, 2, 4]]
        tot[3] = max(tot[3], st[3])
    return {"rays": int(tot[0]), "rays_off_by_1e-3": int(tot[1]), "rays_with_opaque_sample": int(tot[2]),
            "max_rel_error": float(tot[3]), "samples": int(tot[4])}


def test_reverse_reconstruction_of_transmittance():
    ph = config_phantom("diff")
    vol = np.clip((ph.volume.astype(np.float32) + 1024.0) / 4095.0, 0.0, 1.0).astype(np.float32)
    rng = np.random.Generator(np.random.PCG64(1337))
    lut = make_tf_lut(make_tf_control_points(rng))
    views = [dvr.dvr_params(256, 256, view_camera(a), (256, 256, 256), (1, 1, 1), 0.5, 1e-4, 256)
             for a in np.arange(8) * 45.0]
    s = stats(vol, lut, views)
    print(f"benchmark LUT: {s}")
    assert s["rays"] > 0 and s["samples"] > s["rays"]
    # the same workload with every entry above about 580 HU (the spheres) opaque
    opaque = lut.copy()
    opaque[100:, 3] = 1.0
    s2 = stats(vol, opaque, views)
    print(f"LUT with opaque entries: {s2}")
    assert s2["rays_with_opaque_sample"] > 0
