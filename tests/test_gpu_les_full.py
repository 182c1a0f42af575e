"""The learned closure's a-posteriori test at the configuration the closure is
built for: 128^3 LES against box-filtered 512^3 DNS, forced, Re 3000.

The DNS spins up, supplies training snapshots (exact subgrid stress of the
filtered field, every 4th point per axis), the network trains on the GPU, and
LES runs from the filtered DNS state with the learned closure, with the
reference's Smagorinsky model (Cs = 0.18, m_les.f90:1142-1215) and with no
model; each is compared with the filtered DNS spectrum over the window.  The
learned closure must do at least as well as Smagorinsky, and both better than
no model.  About two minutes on one B200."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_learned_les_128_vs_filtered_dns_512():
    from hit3d_b200.les import LesExperiment, run_experiment
    ex = LesExperiment(n_dns=512, n_les=128, re=3000.0, dt_dns=0.00025, nruns=1, spinup=1.5, collect=0.5, nsnap=4,
                       window=1.0, nsample=5, stride=4, train_steps=2000)
    r = run_experiment(ex, log=lambda *a: None)
    err = r["spectrum_error"]
    print(f"512^3 -> 128^3 mean |ln E_LES / E_fDNS|: learned {err['learned']:.4f}, "
          f"Smagorinsky {err['smagorinsky']:.4f}, no model {err['none']:.4f}")
    assert np.isfinite(err["learned"])
    assert err["learned"] <= err["smagorinsky"]
    assert err["smagorinsky"] < err["none"]
