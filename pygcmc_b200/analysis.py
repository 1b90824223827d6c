"""Sampling statistics from the per-step logs: fragment counts and running
energy series, integrated autocorrelation times and decorrelated samples.

The integrated autocorrelation time of a series x_t is
    tau = 1 + 2 sum_{t=1}^{M} rho(t)
with the normalised autocorrelation rho from an FFT and the window M chosen
by Sokal's rule (the smallest M with M >= c tau(M), c = 5); n / tau is the
number of effectively independent samples of a run of n steps.
"""
import numpy as np


def count_series(logs, initial_counts):
    """Total fragment count after each step (all types) from the step logs."""
    counts = np.array(initial_counts, dtype=np.int64).copy()
    out = np.empty(len(logs), dtype=np.int64)
    ftype = logs["ftype"]
    n_after = logs["n_after"]
    move = logs["move"]
    for t in range(len(logs)):
        if move[t] >= 0:
            counts[ftype[t]] = n_after[t]
        out[t] = counts.sum()
    return out


def autocorrelation(x):
    x = np.asarray(x, dtype=np.float64)
    x = x - x.mean()
    n = len(x)
    if n < 2 or not np.any(x):
        return np.ones(1)
    f = np.fft.rfft(x, 2 * n)
    acf = np.fft.irfft(f * np.conj(f))[:n]
    return acf / acf[0]


def integrated_time(x, c: float = 5.0):
    """Integrated autocorrelation time (in steps) with Sokal's window; 1 for a
    constant series."""
    rho = autocorrelation(x)
    if len(rho) == 1:
        return 1.0
    taus = 2.0 * np.cumsum(rho) - 1.0
    m = np.arange(len(taus))
    ok = m >= c * taus
    w = int(np.argmax(ok)) if ok.any() else len(taus) - 1
    return float(max(taus[w], 1.0))


def sampling_summary(logs, initial_counts, steps_per_s: float, burn: int = 0):
    """Acceptance and decorrelation figures of a logged run."""
    L = logs[burn:]
    N = count_series(logs, initial_counts)[burn:]
    E = L["e_total"]
    tau_n, tau_e = integrated_time(N), integrated_time(E)
    tau = max(tau_n, tau_e)
    tr = np.isin(L["move"], [2, 3])
    k = L["k"][tr].sum()
    acc = L["n_accept"][tr].sum()
    return {"steps": int(len(L)), "tau_N": tau_n, "tau_E": tau_e, "tau": tau,
            "decorrelated_samples": len(L) / tau,
            "decorrelated_samples_per_s": steps_per_s / tau,
            "trn_rot_accept_per_pose": float(acc / k) if k else 0.0,
            "trn_rot_accepted_moves_per_step": float(acc / max(1, tr.sum())),
            "mean_N": float(N.mean()), "mean_E": float(E.mean())}
