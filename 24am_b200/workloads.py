"""Seeded synthetic inputs for the AM solver (the benchmark workloads).

The low-rank-plus-noise data matrix stands in for the datasets the reference
was run on (its faces dataset is not shipped):
    D = sum_{k<r} sigma_k u_k v_k^T + N(0, noise^2),  sigma_k = 10 * 0.8^k,
    u_k ~ N(0, I_n) / ||.||,  v_k with nnz_v uniform random indices of N(0, 1)
    values, normalised;  columns centred.
Starting points are i.i.d. U[-1, 1] (density 1), each normalised.
Layout is the reference's: n samples x p features, column-major (as the
reference's m x n matrix B with ldB = m).
"""
import numpy as np


def low_rank_data(n, p, r, nnz_v, seed, noise=0.1, dtype=np.float64):
    """numpy version, n x p column-major."""
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((n, p)) * noise
    for k in range(r):
        u = rng.standard_normal(n)
        u /= np.linalg.norm(u)
        v = np.zeros(p)
        idx = rng.choice(p, size=min(nnz_v, p), replace=False)
        v[idx] = rng.standard_normal(idx.size)
        v /= np.linalg.norm(v)
        # the rank-one term touches only the loading's non-zero columns (adding
        # its zero columns would leave D unchanged)
        D[:, idx] += 10.0 * 0.8 ** k * np.outer(u, v[idx])
    D -= D.mean(axis=0, keepdims=True)
    return np.asfortranarray(D.astype(dtype))


def uniform_starts(p, k, seed, dtype=np.float64):
    """numpy version, p x k column-major."""
    rng = np.random.default_rng(seed)
    V = rng.uniform(-1.0, 1.0, size=(p, k))
    V /= np.linalg.norm(V, axis=0, keepdims=True)
    return np.asfortranarray(V.astype(dtype))


def low_rank_data_torch(n, p, r, nnz_v, seed, noise=0.1, device="cuda"):
    """Same distribution generated on the device in FP32 (benchmark sizes).
    Returns a (p, n) contiguous tensor, i.e. the n x p matrix column-major."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    Dt = torch.randn((p, n), generator=g, device=device, dtype=torch.float32) * noise
    for k in range(r):
        u = torch.randn(n, generator=g, device=device, dtype=torch.float32)
        u /= u.norm()
        idx = torch.randperm(p, generator=g, device=device)[: min(nnz_v, p)]
        vals = torch.randn(idx.numel(), generator=g, device=device, dtype=torch.float32)
        vals /= vals.norm()
        Dt[idx] += (10.0 * 0.8 ** k) * vals[:, None] * u[None, :]
    Dt -= Dt.mean(dim=1, keepdim=True)
    return Dt.contiguous()


def uniform_starts_torch(p, k, seed, device="cuda"):
    """(k, p) contiguous tensor: p x k column-major, unit columns."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    V = torch.rand((k, p), generator=g, device=device, dtype=torch.float32) * 2.0 - 1.0
    V /= V.norm(dim=1, keepdim=True)
    return V.contiguous()


def penalty_gammas(col_norm2_max, col_norm1_max, c=0.1):
    """gamma per penalized formulation: c * max_i ||d_i||_2 for the L2-variance
    forms, c * max_i ||d_i||_1 for the L1-variance forms (the reference compares
    v^2 with gamma for the L0 penalty and |v| for the L1 penalty)."""
    return {4: c * col_norm2_max, 6: c * col_norm2_max, 5: c * col_norm1_max,
            7: c * col_norm1_max}
