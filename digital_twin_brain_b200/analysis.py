"""Long-run spike statistics used to compare closed-loop runs
(analysis/spike_statistics.py and analysis/getpsd.py, restated; spike
rasters are [time, neuron] arrays as the reference expects).

Chaotic spiking networks diverge after the first float-rounding difference,
so a push-mode run (float atomics) and a reference run agree in these
statistics, not spike by spike; the pull path reproduces them exactly.
"""
from __future__ import annotations

import numpy as np
from scipy.ndimage import uniform_filter1d
from scipy.signal import get_window, welch


def mean_firing_rate(spike_train: np.ndarray) -> float:
    """analysis/spike_statistics.py:8-24: mean over neurons whose mean exceeds 0.001 (if more than 10)."""
    active = np.where(spike_train.mean(axis=0) > 0.001)[0]
    if len(active) > 10:
        return float(np.mean(spike_train[:, active]))
    return 0.0


def instantaneous_rate(spike_train: np.ndarray, bin_width: int = 5) -> np.ndarray:
    """analysis/spike_statistics.py:27-42: population mean per step, box-filtered."""
    return uniform_filter1d(spike_train.mean(axis=1).astype(np.float32), size=bin_width)


def spike_psd(spike_train: np.ndarray, sampling_rate: float = 1000, subtract_mean: bool = False):
    """analysis/spike_statistics.py:64-80: |rfft|^2 of the instantaneous rate."""
    st = instantaneous_rate(spike_train, bin_width=5)
    data = st - np.mean(st) if subtract_mean else st
    power = np.square(np.abs(np.fft.rfft(data)))
    return np.linspace(0, sampling_rate / 2, len(power)), power


def coefficient_of_variation(spike_train: np.ndarray) -> float:
    """analysis/spike_statistics.py:114-124: mean ISI CV of neurons with more than 5 spikes (NaN if < 10)."""
    active = (spike_train.sum(0) > 5).nonzero()[0]
    if len(active) < 10:
        return float("nan")
    cvs = []
    for i in active:
        t = spike_train[:, i].nonzero()[0]
        isi = t[1:] - t[:-1]
        cvs.append(isi.std() / isi.mean())
    return float(np.mean(cvs))


def get_psd(data: np.ndarray, fs: float, resolution: float = 0.5):
    """analysis/getpsd.py:9-19: Welch PSD with a boxcar window of fs/resolution samples, 75 % overlap."""
    win = int(fs / resolution)
    return welch(data, fs=fs, window=get_window("boxcar", win), noverlap=int(0.75 * win), nfft=win, axis=0,
                 scaling="density", detrend=False)
