"""The full-model pipeline on the GPU at a small size: the learned-opacities
disk (surrogate opacities, mixed precision) iterated to hydrostatic
equilibrium with settling recomputed every pass, its spectra and images,
the same pipeline in the FP64 form with DHS opacities, and the mixed
pipeline again with another seed (the noise floor of the comparison)."""
import numpy as np
import pytest

from mcmax_b200 import full_model as F

pytestmark = pytest.mark.gpu


def test_full_model_pipeline_small(tmp_path):
    res = F.main(["--nrad", "24", "--ntheta", "20", "--nlam", "40", "--nphot", "2e5", "--passes", "2",
                  "--npix", "32", "--nint", "20", "--angles", "20,80", "--image-lam", "10", "--check", "--floor",
                  "--out", str(tmp_path)])
    for arm in ("mixed_surrogate", "fp64_dhs"):
        r = res[arm]
        assert len(r["packet_runs"]) == 3 and all(p["packets"] == 200000 for p in r["packet_runs"])
        assert len(r["errT"]) == 2 and all(np.isfinite(r["errT"]))
        assert r["timings_s"]["structure_s"] > 0
    assert res["mixed_surrogate"]["bins_served_by_network"] > 0
    ag, fl = res["agreement"], res["noise_floor"]
    print("agreement", ag)
    print("floor", fl)
    assert ag["cells_nabs_ge_1e3"] > 20
    # the FP64 + DHS pipeline differs from the mixed one by little more
    # than a second seed of the mixed one does
    assert ag["T_median_rel"] < 2.0 * fl["T_median_rel"] + 0.01
    for k, s in ag["spectra"].items():
        assert s["wavelengths"] > 10 and s["median_rel"] < 2.0 * fl["spectra"][k]["median_rel"] + 0.02
    for im in ag["images"].values():
        assert 0.9 < im["total_flux_ratio"] < 1.1
    assert len(res["files"]) == 1 + 2 + 2
