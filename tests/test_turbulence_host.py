"""Host-side parts of the decaying-turbulence case (no GPU): the seeded start field and the
spectrum tools."""
import numpy as np

from periodicshiftlbm_b200.turbulence import box_filter, energy_spectrum, initial_velocity, spectrum_error


def test_start_field_is_divergence_free_and_scaled():
    M = 32
    u = initial_velocity(M, seed=3)
    assert u.shape == (3, M, M, M) and u.dtype == np.float32
    assert abs(np.sqrt(np.mean(u.astype(np.float64) ** 2)) - 0.04) < 1e-6
    uh = np.fft.rfftn(u.astype(np.float64), axes=(1, 2, 3))
    kz = np.fft.fftfreq(M, 1.0 / M)[:, None, None]
    ky = np.fft.fftfreq(M, 1.0 / M)[None, :, None]
    kx = np.fft.rfftfreq(M, 1.0 / M)[None, None, :]
    div = kx * uh[0] + ky * uh[1] + kz * uh[2]
    assert np.max(np.abs(div)) < 1e-5 * np.max(np.abs(uh))  # float32 field, Nyquist planes
    assert np.array_equal(u, initial_velocity(M, seed=3))


def test_spectrum_peaks_near_k0_and_holds_the_energy():
    M = 64
    u = initial_velocity(M, seed=1).astype(np.float64)
    k, E = energy_spectrum(u)
    assert abs(E.sum() - 0.5 * np.mean((u ** 2).sum(0))) < 1e-9
    assert 2 <= int(np.argmax(E)) <= 6
    assert spectrum_error(E, E, 20) == 0.0


def test_box_filter_averages_blocks():
    u = np.arange(2 * 4 * 4 * 4, dtype=np.float64).reshape(2, 4, 4, 4)
    f = box_filter(u)
    assert f.shape == (2, 2, 2, 2)
    assert f[0, 0, 0, 0] == u[0, :2, :2, :2].mean()
