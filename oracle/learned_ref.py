"""CPU reference of the learned-preconditioner training objective -- TEST
INFRASTRUCTURE ONLY.  Written independently of the GPU kernels in torch
(float64, CPU) so that its gradient comes from automatic differentiation,
against which the GPU's hand-written backward pass is checked.

Objective (see rpba_b200/csrc/learned.cu): per system and right-hand side b,
with C = blockdiag(diag(s_k) Sinv_k diag(s_k)), u = C b + uc (uc: the fixed
coarse-space part of the preconditioned right-hand side), v = S u,
loss = ln(u^T v) - 2 ln(b^T u), averaged over systems and right-hand sides;
s_k = exp(tanh(W2 tanh(W1 f_k + b1) + b2)) on the block's parameters.
"""
import numpy as np

NN_F, NN_H, NN_O = 19, 64, 9


def loss(ts: dict, weights: np.ndarray):
    """Returns (loss, gradient) as numpy arrays."""
    import torch
    W = torch.tensor(np.asarray(weights, np.float64), requires_grad=True)
    W1 = W[: NN_H * NN_F].reshape(NN_H, NN_F)
    b1 = W[NN_H * NN_F: NN_H * NN_F + NN_H]
    o2 = NN_H * NN_F + NN_H
    W2 = W[o2: o2 + NN_O * NN_H].reshape(NN_O, NN_H)
    b2 = W[o2 + NN_O * NN_H:]
    R, P = int(ts["rows"]), int(ts["probes"])
    f = torch.tensor(np.asarray(ts["features"], np.float64).reshape(R, NN_F))
    h = torch.tanh(f @ W1.T + b1)
    s = torch.exp(torch.tanh(h @ W2.T + b2))
    npar = np.asarray(ts["np"])
    mask = torch.tensor((np.arange(9)[None, :] < npar[:, None]).astype(np.float64))
    s = s * mask + (1 - mask)
    Si = torch.tensor(np.asarray(ts["sinv"], np.float64).reshape(R, 9, 9))
    b = torch.tensor(np.asarray(ts["b"], np.float64).reshape(P, R, 9))
    u = s[None] * torch.einsum("rac,prc->pra", Si, s[None] * b)
    if ts.get("uc") is not None:
        u = u + torch.tensor(np.asarray(ts["uc"], np.float64).reshape(P, R, 9))
    # v = S u over the block rows
    blocks = torch.tensor(np.asarray(ts["blocks"], np.float64).reshape(-1, 9, 9))
    rowoff = np.asarray(ts["rowoff"])
    col = np.asarray(ts["ent_col"])
    blk = np.asarray(ts["ent_blk"]).astype(np.int64) & 0xFFFFFFFF
    tr = (blk & 0x80000000) != 0
    bi = blk & 0x7FFFFFFF
    rows = np.repeat(np.arange(R), np.diff(rowoff))
    Bm = blocks[bi]
    Bm = torch.where(torch.tensor(tr)[:, None, None], Bm.transpose(1, 2), Bm)
    contrib = torch.einsum("eac,pec->pea", Bm, u[:, col])
    v = torch.zeros_like(u).index_add_(1, torch.tensor(rows), contrib)
    sys = np.asarray(ts["sys"])
    S = int(ts["systems"])
    st = torch.tensor(sys)
    pp = torch.zeros(P, S, dtype=torch.float64).index_add_(1, st, (b * u).sum(-1))
    qq = torch.zeros(P, S, dtype=torch.float64).index_add_(1, st, (u * v).sum(-1))
    L = (torch.log(qq) - 2 * torch.log(pp)).mean()
    L.backward()
    return float(L.detach()), W.grad.numpy().copy()


def random_set(rng, systems=3, rows_per=12, probes=2, density=0.3):
    """A random training set: SPD block systems scaled to unit diagonal."""
    feats, sinv, bs, xs, nps, sysv, rowoff, ec, eb, blocks, sys_row = [], [], [], [], [], [], [0], [], [], [], [0]
    row0 = 0
    for sy in range(systems):
        n = rows_per
        npar = rng.choice([9, 8, 9, 3], size=n)
        npar[0] = 9
        M = np.zeros((9 * n, 9 * n))
        mask = np.zeros((9 * n,), bool)
        for k in range(n):
            mask[9 * k: 9 * k + npar[k]] = True
        A = rng.normal(size=(9 * n, 9 * n)) * (rng.random((n, n)) < density).repeat(9, 0).repeat(9, 1)
        M = A @ A.T + 9 * n * 0.3 * np.eye(9 * n)
        M[~mask, :] = 0
        M[:, ~mask] = 0
        M[~mask, ~mask] = 1.0
        d = np.sqrt(np.diag(M))
        Ms = M / d[:, None] / d[None, :]
        Ms[~mask, ~mask] = 1.0
        base_blk = len(blocks)
        for k in range(n):
            Dk = Ms[9 * k: 9 * k + 9, 9 * k: 9 * k + 9].copy()
            Dk[npar[k]:, :] = 0
            Dk[:, npar[k]:] = 0
            inv = np.zeros((9, 9))
            q = npar[k]
            inv[:q, :q] = np.linalg.inv(Dk[:q, :q])
            sinv.append(inv)
            blocks.append(Dk)
        pairs = {}
        for k in range(n):
            for l in range(k + 1, n):
                B = Ms[9 * k: 9 * k + 9, 9 * l: 9 * l + 9]
                if np.abs(B).max() > 0:
                    pairs[(k, l)] = len(blocks)
                    blocks.append(B.copy())
        for k in range(n):
            ents = []
            for l in range(n):
                if l < k and (l, k) in pairs:
                    ents.append((row0 + l, pairs[(l, k)] | 0x80000000))
                elif l == k:
                    ents.append((row0 + k, base_blk + k))
                elif l > k and (k, l) in pairs:
                    ents.append((row0 + l, pairs[(k, l)]))
            for c, bb in ents:
                ec.append(c)
                eb.append(np.int64(bb).astype(np.int32) if bb < 2 ** 31 else np.int32(bb - 2 ** 32))
            rowoff.append(rowoff[-1] + len(ents))
            feats.append(rng.normal(size=NN_F))
            nps.append(npar[k])
            sysv.append(sy)
        bsys = rng.normal(size=(probes, 9 * n)) * mask
        x0 = np.linalg.lstsq(Ms, bsys[0], rcond=None)[0] * mask
        bs.append(bsys.reshape(probes, n, 9))
        xs.append(x0.reshape(n, 9))
        row0 += n
        sys_row.append(row0)
    return {"rows": row0, "systems": systems, "probes": probes, "features": np.array(feats, np.float32),
            "sinv": np.array(sinv, np.float32), "b": np.concatenate(bs, axis=1).astype(np.float32),
            "xs": np.concatenate(xs).astype(np.float32), "np": np.array(nps, np.int32),
            "sys": np.array(sysv, np.int32), "rowoff": np.array(rowoff, np.int32),
            "ent_col": np.array(ec, np.int32), "ent_blk": np.array(eb, np.int32),
            "blocks": np.array(blocks, np.float32), "sys_row": np.array(sys_row, np.int32)}
