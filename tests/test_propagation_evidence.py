"""metrics(result) / verify(result) evidence over saved spectra -- CPU only.

The field-metric restatement is pinned on the reference's known answers
(test/core/test_numerical_kernels.jl:266-273), and metrics/verify are driven
over spectra saved by the FP64 oracle the way test/core/test_propagation.jl:
62-111 drives them over a propagate result (the GPU result gets the same
checks in tests/test_gpu_parity.py).
"""
import numpy as np
import pytest

from fiberlab_gpu import problem as P
from fiberlab_gpu import solve as S
from oracle import oracle as O


def test_field_metric_known_answers():
    # test_numerical_kernels.jl:266-273
    nt = 64
    sim = P.get_disp_sim_params(1550e-9, 1, nt, 10.0, 2)
    constant = S.field_metrics(np.fft.ifft(np.ones(nt))[None, :], sim)
    impulse_t = np.zeros(nt, complex)
    impulse_t[nt // 2] = 1
    impulse = S.field_metrics(np.fft.ifft(impulse_t)[None, :], sim)
    assert constant["temporal_edge_fraction"] == pytest.approx(6 / nt, rel=1e-12)
    assert constant["spectral_edge_fraction"] < 1e-30
    assert impulse["temporal_edge_fraction"] < 1e-30
    assert impulse["spectral_edge_fraction"] == pytest.approx(6 / nt, rel=1e-12)
    assert S.edge_fraction(np.ones(10)) == 0.2
    with pytest.raises(P.ArgumentError):
        S.edge_fraction(np.zeros(8))


def _oracle_result(fp, zs):
    spectra, st, _ = O.forward(fp, zsave=zs)
    spectra = np.asarray(spectra)
    return S.PropagationResult(z_m=np.asarray(zs, dtype=float), spectra=spectra,
                               input_spectrum=spectra[0].copy(),
                               output_spectrum=spectra[-1].copy(),
                               accepted_steps=st["naccept"], rhs_evaluations=st["nf"],
                               problem=fp)


def test_metrics_and_verify_over_saved_spectra():
    # the reference test's shape (test_propagation.jl:19-33): SMF-28 with β2
    # only, 0.1 mm, 10 µW, 250 fs Gaussian at 50 MHz, 128 samples over 3 ps
    fp = P.single_mode_problem(nt=128, time_window_ps=3.0, L=1e-4, power_w=1e-5,
                               fwhm_s=250e-15, rep_rate_hz=50e6, pulse="gauss",
                               betas=(-2.17e-26,), beta_order=2)
    res = _oracle_result(fp, [0.0, 0.5e-4, 1e-4])
    ev = S.metrics(res)
    assert ev["samples"] == 128 and ev["modes"] == 1 and ev["saved_positions"] == 3
    assert ev["input_energy_pj"] == pytest.approx(1e-5 / 50e6 * 1e12, rel=1e-5)
    assert ev["output_energy_pj"] > 0 and ev["output_peak_power_w"] > 0
    assert len(ev["output_mode_energy_pj"]) == 1
    assert ev["launch_samples_per_fwhm"] == pytest.approx(250e-15 * 1e12 / fp.sim["Δt"])
    assert ev["max_photon_number_drift"] < 1e-8
    v = S.verify(res)
    assert v["pass"] and v["integrity_ok"] and v["finite_fields"]
    assert v["temporal_edges_contained"] and v["spectral_edges_contained"]
    assert v["launch_sampling_ok"] and v["photon_number_conserved"]
    assert not S.verify(res, min_launch_samples_per_fwhm=16)["pass"]
    assert S.verify(res, photon_drift_limit=None)["photon_number_conserved"] is None
    assert S.verify(res, energy_drift_limit=1.0)["energy_change_acceptable"]
    with pytest.raises(P.ArgumentError):
        S.verify(res, temporal_edge_limit=2.0)
    # a mutated result fails integrity with the same keys, and metrics refuses it
    res.spectra[-1, 0, 0] += 1.0
    bad = S.verify(res)
    assert not bad["pass"] and not bad["integrity_ok"]
    assert bad.keys() == v.keys() and bad["max_photon_number_drift"] is None
    with pytest.raises(P.ArgumentError):
        S.metrics(res)
