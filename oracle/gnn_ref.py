"""FP64 restatement of the learned-FSAI network (mphyfem_b200/csrc/gnn.cu) with torch autograd on
the CPU. Test infrastructure only: the checker for the GPU forward and backward kernels.

Features follow the GPU: A^ = D^{-1/2} A D^{-1/2} with prescribed DOFs as identity rows; node
input = A^_nn (9), prescribed flags (3), (neighbours - 1) / 27; edge input = A^_nm (off-diagonal
blocks); prediction base_n P with base_n the block-Jacobi FSAI block; loss Kaporin's condition
number of G^ A^ G^T (dense, small problems only). Weights are rounded to BF16 as on the GPU.
"""
from __future__ import annotations

import numpy as np
import torch

H, L, NIN = 64, 3, 13


def layout():
    off = {}
    o = 0

    def add(name, n):
        nonlocal o
        off[name] = (o, n)
        o += n
    add("w_in", H * NIN)
    add("b_in", H)
    for l in range(L):
        add(f"U{l}", H * H)
        add(f"V{l}", H * 9)
        add(f"c{l}", H)
        add(f"S{l}", H * H)
        add(f"T{l}", H * H)
        add(f"d{l}", H)
    add("Wa", 9 * H)
    add("Wb", 9 * H)
    add("Wc", 81)
    add("bo", 9)
    return off, o


def loss_and_grads(params, A_full, fixed, nbrs, lrow, lcol):
    """params: flat float32; A_full: scipy node-major operator; nbrs: ascending neighbour lists;
    (lrow, lcol): lower pattern. Loss: Kaporin's log K of G^ A^ G^T up to the constant
    (1/N) log det A^, i.e. log(tr(G^ A^ G^T) / N) - (2/N) sum_n log|det G^_nn| (N = 3 n_node).
    Returns (loss, flat gradient, predicted unscaled blocks)."""
    off, total = layout()
    p32 = torch.tensor(np.asarray(params, np.float32))
    pb = p32.to(torch.bfloat16).to(torch.float64).detach().requires_grad_(True)

    def W(name, shape):
        o, n = off[name]
        return pb[o:o + n].view(*shape)

    A = A_full.tocsr()
    n_node = len(nbrs)
    d = np.abs(A.diagonal())
    s = np.where(d > 0, np.sqrt(d), 1.0)
    fx = np.asarray(fixed).reshape(-1, 3).astype(np.float64)

    def blk(n, m):
        b = A[3 * n:3 * n + 3, 3 * m:3 * m + 3].toarray()
        return b / np.outer(s[3 * n:3 * n + 3], s[3 * m:3 * m + 3])

    x = np.zeros((n_node, NIN))
    src, dst, e = [], [], []
    for n in range(n_node):
        x[n, :9] = blk(n, n).ravel()
        x[n, 9:12] = fx[n]
        x[n, 12] = (len(nbrs[n]) - 1) / 27.0
        for m in nbrs[n]:
            if m != n:
                src.append(m)
                dst.append(n)
                e.append(blk(n, m).ravel())
    deg = torch.tensor(np.maximum(np.array([len(nb) - 1 for nb in nbrs]), 1), dtype=torch.float64)
    X = torch.tensor(x)
    src_t, dst_t = torch.tensor(src), torch.tensor(dst)
    E = torch.tensor(np.array(e))
    h = torch.relu(X @ W("w_in", (H, NIN)).T + W("b_in", (H,)))
    for l in range(L):
        P = h @ W(f"U{l}", (H, H)).T
        pre = P[src_t] + E @ W(f"V{l}", (H, 9)).T + W(f"c{l}", (H,))
        msg = torch.zeros_like(h).index_add_(0, dst_t, torch.relu(pre)) / deg[:, None]
        q = h @ W(f"S{l}", (H, H)).T + msg @ W(f"T{l}", (H, H)).T + W(f"d{l}", (H,))
        h = h + torch.relu(q)
    rows = np.repeat(np.arange(n_node), np.diff(lrow))
    # the edge term acts on off-diagonal blocks only
    el = torch.tensor(np.array([blk(n, m).ravel() if n != m else np.zeros(9) for n, m in zip(rows, lcol)]))
    out = (h[torch.tensor(rows)] @ W("Wa", (9, H)).T + h[torch.tensor(lcol.astype(np.int64))] @ W("Wb", (9, H)).T
           + el @ W("Wc", (9, 9)).T + W("bo", (9,)))
    # the prediction is base_n P with P = decoder + [n == m] I, base_n the block-Jacobi FSAI
    # (gnn.cu base_kernel): G_nn = L^T, L L^T = (A^_nn)^-1
    base_node = np.zeros((n_node, 3, 3))
    for n in range(n_node):
        B = blk(n, n)
        B = 0.5 * (B + B.T)
        g = np.eye(3)
        if np.linalg.det(B) > 0:
            try:
                g = np.linalg.cholesky(np.linalg.inv(B)).T
            except np.linalg.LinAlgError:
                g = np.eye(3)
        base_node[n] = g
    eye_rows = np.array([np.eye(3).ravel() if n == m else np.zeros(9) for n, m in zip(rows, lcol)])
    P = (out + torch.tensor(eye_rows)).view(-1, 3, 3)
    out = torch.bmm(torch.tensor(base_node[rows]), P).reshape(-1, 9)
    # entries with a prescribed row or column DOF are fixed to the identity (gnn.cu dec_fwd)
    keep = np.ones((len(rows), 3, 3))
    ident = np.zeros((len(rows), 3, 3))
    for j, (n, m) in enumerate(zip(rows, lcol)):
        keep[j] = 1.0 - np.maximum(fx[n][:, None], fx[m][None, :])
        if n == m:
            ident[j] = np.diag(fx[n])
    keep_t, ident_t = torch.tensor(keep.reshape(-1, 9)), torch.tensor(ident.reshape(-1, 9))
    out = out * keep_t + ident_t
    scol = torch.tensor(np.stack([s[3 * m:3 * m + 3] for m in lcol]))          # [n_lower, 3]
    N = 3 * n_node
    Gd = torch.zeros((N, N), dtype=torch.float64)
    blocks = out.view(-1, 3, 3)
    for j, (n, m) in enumerate(zip(rows, lcol)):
        Gd[3 * n:3 * n + 3, 3 * m:3 * m + 3] = blocks[j]
    Ah = np.zeros((N, N))
    for n in range(n_node):
        for m in nbrs[n]:
            Ah[3 * n:3 * n + 3, 3 * m:3 * m + 3] = blk(n, m)
    tr = torch.trace(Gd @ torch.tensor(Ah) @ Gd.T)
    diag = [j for j, (n, m) in enumerate(zip(rows, lcol)) if n == m]
    logdet = sum(torch.log(torch.abs(torch.det(blocks[j]))) for j in diag)
    loss = torch.log(tr / N) - 2.0 / N * logdet
    loss.backward()
    pred = (blocks / scol[:, None, :]).detach().numpy()
    return float(loss.detach()), pb.grad.numpy().copy(), pred
