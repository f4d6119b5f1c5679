"""CPU checks of the policy-fused kernel's network layout (no GPU).

The fused kernel reads its operands through tcgen05 shared-memory matrix
descriptors in the no-swizzle K-major layout: an operand of R rows is a grid
of 8x8 BF16 core matrices (128 contiguous bytes, rows 16 bytes apart), the
next core matrix along K `LBO` bytes away and the next 8-row group `SBO`
bytes away.  These tests replay, in numpy, exactly the descriptor start
addresses, LBO and SBO that the kernel issues (g1_mlp.cuh, Runner::issue,
tile_off) against the bytes that pack_weights produces and the A tile that
the epilogue writes, and check the products equal x @ W^T of every layer.
"""
import numpy as np
import torch

from g1sim_b200 import policy as P

ROWS = 128
STAGE = 16384


def tile_off(row, k, R=ROWS):
    """Byte offset of (row, k) in an A tile (g1_mlp.cuh tile_off)."""
    return ((k >> 3) * (R >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2


def desc_read(buf, start, lbo, sbo, rows, k=16):
    """Elements (r, k) of the 16-wide K slice a descriptor addresses:
    start + (r // 8) * SBO + (r % 8) * 16 + (k // 8) * LBO + (k % 8) * 2."""
    r = np.arange(rows)[:, None]
    kk = np.arange(k)[None, :]
    off = start + (r // 8) * sbo + (r % 8) * 16 + (kk // 8) * lbo + (kk % 8) * 2
    return buf[off // 2]


def bf16_bits(t):
    return t.to(torch.bfloat16).view(torch.int16).numpy().astype(np.uint16)


def bits_to_f32(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


def layer_via_descriptors(a_tile_u16, blob_u16, blob_off_bytes, K, N, KC):
    """D = A W^T the way Runner::issue walks chunks, K steps and N halves."""
    lbo_a, lbo_b = ROWS * 16, N * 16
    nmma = N // 256 if N > 256 else 1
    nn = 256 if N > 256 else N
    chunk_bytes = N * KC * 2
    D = np.zeros((ROWS, N), np.float64)
    for c in range(K // KC):
        stage = blob_u16[(blob_off_bytes + c * chunk_bytes) // 2:(blob_off_bytes + (c + 1) * chunk_bytes) // 2]
        for j in range(KC // 16):
            kk = c * (KC // 16) + j
            a = bits_to_f32(desc_read(a_tile_u16, kk * 2 * lbo_a, lbo_a, 128, ROWS)).astype(np.float64)
            for h in range(nmma):
                b = bits_to_f32(desc_read(stage, j * 2 * lbo_b + h * 32 * 128, lbo_b, 128, nn)).astype(np.float64)
                D[:, h * 256:h * 256 + nn] += a @ b.T
    return D


def make_a_tile(x, K):
    """A tile bytes as the kernel's st_row8 writes them (x: ROWS x K float)."""
    bits = bf16_bits(torch.as_tensor(x, dtype=torch.float32))
    tile = np.zeros(ROWS * K, np.uint16)
    for row in range(ROWS):
        for k in range(K):
            tile[tile_off(row, k) // 2] = bits[row, k]
    return tile


def test_chunks_fit_stages_and_sizes_add_up():
    total = 0
    for net in ("critic", "actor"):
        for fin, fout, kp, np_, kc in P._LAYERS[net]:
            assert np_ * kc * 2 <= STAGE and kp % kc == 0 and kc % 16 == 0 and np_ % 16 == 0
            assert kp >= fin and np_ >= fout
            total += np_ * kp * 2
    ac = P.ActorCritic()
    wb, bb = P.pack_weights(ac)
    assert wb.numel() * 2 == total
    assert bb.numel() == 512 + 256 + 128 + 16 + 512 + 256 + 128 + 32


def test_descriptor_walk_reproduces_every_layer():
    torch.manual_seed(0)
    ac = P.ActorCritic().xavier_(torch.Generator().manual_seed(1))
    for m in ac.modules():
        if isinstance(m, torch.nn.Linear):
            torch.nn.init.uniform_(m.bias, -0.1, 0.1)
    wb, bb = P.pack_weights(ac)
    blob = wb.view(torch.int16).numpy().astype(np.uint16)
    off = 0
    for net in ("critic", "actor"):
        lins = P._linears(getattr(ac, net))
        for lin, (fin, fout, kp, np_, kc) in zip(lins, P._LAYERS[net]):
            x = np.zeros((ROWS, kp), np.float32)
            x[:, :fin] = np.random.default_rng(fin + fout).normal(size=(ROWS, fin))
            D = layer_via_descriptors(make_a_tile(x, kp), blob, off, kp, np_, kc)
            xb = bits_to_f32(bf16_bits(torch.tensor(x))).astype(np.float64)
            wbf = bits_to_f32(bf16_bits(lin.weight.detach())).astype(np.float64)
            ref = xb[:, :fin] @ wbf.T
            np.testing.assert_allclose(D[:, :fout], ref, rtol=1e-12, atol=1e-12)
            assert np.all(D[:, fout:] == 0.0)
            off += np_ * kp * 2


def test_bias_blob_layout():
    ac = P.ActorCritic()
    for i, m in enumerate(ac.modules()):
        if isinstance(m, torch.nn.Linear):
            torch.nn.init.constant_(m.bias, float(i))
    _, bb = P.pack_weights(ac)
    o = 0
    for net in ("critic", "actor"):
        for lin, (fin, fout, kp, np_, kc) in zip(P._linears(getattr(ac, net)), P._LAYERS[net]):
            assert torch.equal(bb[o:o + fout], lin.bias.detach())
            assert torch.all(bb[o + fout:o + np_] == 0)
            o += np_
    assert o == bb.numel()


def test_state_dict_names_match_reference():
    # reference examples/train.py:16-47 module layout
    keys = set(P.ActorCritic().state_dict().keys())
    for net in ("actor", "critic"):
        for i in (0, 2, 4, 6):
            assert f"{net}.{i}.weight" in keys and f"{net}.{i}.bias" in keys
    assert {"std", "obs_mean", "obs_var", "obs_count"} <= keys


def test_gae_matches_reference_recursion():
    g = torch.Generator().manual_seed(3)
    T, n = 6, 5
    r, v = torch.randn(T, n, generator=g), torch.randn(T, n, generator=g)
    d = (torch.rand(T, n, generator=g) < 0.2).float()
    nv, nd = torch.randn(n, generator=g), (torch.rand(n, generator=g) < 0.3)
    ret, adv = P.gae(r, v, d, nv, nd)
    # scalar restatement of reference train.py:104-121
    for e in range(n):
        last = 0.0
        for t in reversed(range(T)):
            nnt = 1.0 - (float(nd[e]) if t == T - 1 else float(d[t + 1, e]))
            nval = float(nv[e]) if t == T - 1 else float(v[t + 1, e])
            delta = float(r[t, e]) + 0.99 * nval * nnt - float(v[t, e])
            last = delta + 0.99 * 0.95 * nnt * last
            assert abs(float(adv[t, e]) - last) < 1e-5
            assert abs(float(ret[t, e]) - (last + float(v[t, e]))) < 1e-5


def test_policy_pt_round_trip(tmp_path):
    ac = P.ActorCritic().xavier_(torch.Generator().manual_seed(4))
    with torch.no_grad():
        ac.obs_mean.uniform_(-1, 1)
        ac.std.fill_(-0.7)
    path = tmp_path / "policy.pt"
    torch.save(ac.state_dict(), path)
    bc = P.load_policy_pt(str(path), device="cpu")
    for (ka, va), (kb, vb) in zip(ac.state_dict().items(), bc.state_dict().items()):
        assert ka == kb and torch.equal(va, vb)
    wa, ba = P.pack_weights(ac)
    wb, bb = P.pack_weights(bc)
    assert torch.equal(wa, wb) and torch.equal(ba, bb)
