"""Seeded synthetic HRRT 64-bit listmode streams, generated on the GPU.

No scanner listmode ships with the reference; the benchmark and the parity
tests draw events like this:

  * coincidences: a head pair (1..20), crystals (x 0..71, y 0..103, with a
    ring difference of at most 40), DOI layers 0/1, drawn uniformly and kept
    with probability E[bin] / max(E), where E is the expected prompt sinogram
    (span 3) of the config-1 phantom -- FP(activity) attenuated by
    exp(-FP(mu)), plus flat randoms at 20 % of the prompts -- and `bin` the
    sinogram bin the event rebins to (a float32 evaluation of rebin_event,
    LM_Rebinner_mp.cpp:188-219, used only for the acceptance weight);
  * 10 % delayed events, drawn uniformly over the LORs that rebin (randoms
    are flat);
  * a time tag (0x80000000 | ms) before every `events_per_ms` events,
    counting milliseconds from 0.

Word layout (histogram_mp.cpp:1026-1233): ew1 = ax | ay<<8 | (mp&7)<<16 |
doia<<22 with top bits 00; ew2 = bx | by<<8 | (mp>>3)<<16 | doib<<22 with top
bits 11 (prompt) or 10 (delayed); a tag is ew1 = 0x4000xxxx, ew2 = 0xC000yyyy
carrying the 32-bit value yyyyxxxx.
"""
import numpy as np

SINO_PLANE = 256 * 288


def expected_prompts(ctx, seed=0, randoms_frac=0.20):
    """Expected prompts (flat-file layout, float32 numpy) of the phantom of
    `seed` on the span of `ctx`: attenuated line integrals plus flat randoms."""
    from hrrt_reconstruction_b200 import phantom
    fp = ctx.forward_project(phantom.phantom(ctx, seed=seed))
    mu = ctx.forward_project(phantom.mu_map(ctx))
    t = fp * np.exp(-mu)
    valid = fp > 0
    r = randoms_frac / (1.0 - randoms_frac) * float(t.sum(dtype=np.float64)) / max(int(valid.sum()), 1)
    return (t + np.float32(r) * valid).astype(np.float32)


class _Tables:
    def __init__(self, torch, dev, span):
        import hrrt_reconstruction_b200 as H
        sol = H.lm_table("sol", span).reshape(-1)
        self.nsino = torch.from_numpy(sol["nsino"].astype(np.int64)).to(dev)
        self.d = torch.from_numpy(sol["d"].copy()).to(dev)
        self.z = torch.from_numpy(sol["z"].copy()).to(dev)
        self.zpos = torch.from_numpy(H.lm_table("zpos", span)).to(dev)
        self.zpos2 = torch.from_numpy(H.lm_table("zpos2", span)).to(dev)
        self.segz0 = torch.from_numpy(H.lm_table("segz0", span).astype(np.int64)).to(dev)
        self.segzmax = torch.from_numpy(H.lm_table("segzmax", span).astype(np.int64)).to(dev)
        self.segzoff = torch.from_numpy(H.lm_table("segzoffset", span).astype(np.int64)).to(dev)


def _candidates(torch, T, g, n, dev, max_rd=40):
    mp = torch.randint(1, 21, (n,), generator=g, device=dev)
    ax = torch.randint(0, 72, (n,), generator=g, device=dev)
    bx = torch.randint(0, 72, (n,), generator=g, device=dev)
    ay = torch.randint(0, 104, (n,), generator=g, device=dev)
    by = (ay + torch.randint(-max_rd, max_rd + 1, (n,), generator=g, device=dev)).clamp_(0, 103)
    la = torch.randint(0, 2, (n,), generator=g, device=dev)
    lb = torch.randint(0, 2, (n,), generator=g, device=dev)
    idx = (mp * 144 + ax + 72 * la) * 144 + bx + 72 * lb
    ns = T.nsino[idx]
    dz2 = T.zpos[by] - T.zpos[ay]
    plane = (T.zpos2[ay] + T.z[idx] * dz2).to(torch.int64)
    seg = 0.5 + dz2 * T.d[idx]
    sn = seg.to(torch.int64)
    segnum = torch.where(seg < 0, 1 - 2 * sn, 2 * sn)
    ok = (ns >= 0) & (segnum < T.segz0.numel()) & (plane >= 0) & (plane <= 206)
    sg = segnum.clamp(0, T.segz0.numel() - 1)
    ok &= (plane >= T.segz0[sg]) & (plane <= T.segzmax[sg])
    addr = torch.where(ok, (plane + T.segzoff[sg]) * SINO_PLANE + ns.clamp(min=0), torch.zeros_like(ns))
    return mp, ax, ay, bx, by, la, lb, ok, addr


def _to_i32(torch, v):
    return torch.where(v >= 2 ** 31, v - 2 ** 32, v).to(torch.int32)


def synth_words(n_events, expected, seed=0, span=3, events_per_ms=1000, delayed_frac=0.10, chunk=1 << 25,
                device="cuda"):
    """-> int32 torch tensor on `device`: the word stream (reinterpret as
    uint32), with n_events coincidences (each delayed with probability
    `delayed_frac`) and a time tag before every `events_per_ms` of them.
    `expected`: flat expected-prompts sinogram (numpy or torch) for the
    acceptance weights."""
    import torch
    dev = torch.device(device)
    T = _Tables(torch, dev, span)
    E = torch.as_tensor(expected, device=dev).reshape(-1).float()
    E = E / E.max()
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))

    def fill(prompt, m):
        parts, have = [], 0
        while have < m:
            mp, ax, ay, bx, by, la, lb, ok, addr = _candidates(torch, T, g, 2 * m, dev)
            keep = ok & (torch.rand(2 * m, generator=g, device=dev) < E[addr]) if prompt else ok
            sel = torch.nonzero(keep).squeeze(1)[: m - have]
            if sel.numel() == 0:
                continue
            top = 0xC0000000 if prompt else 0x80000000
            parts.append((ax[sel] | (ay[sel] << 8) | ((mp[sel] & 7) << 16) | (la[sel] << 22),
                          bx[sel] | (by[sel] << 8) | ((mp[sel] >> 3) << 16) | (lb[sel] << 22) | top))
            have += sel.numel()
        return torch.cat([a for a, _ in parts]), torch.cat([b for _, b in parts])

    ntags = (n_events + events_per_ms - 1) // events_per_ms
    out = torch.empty(2 * (n_events + ntags), dtype=torch.int32, device=dev)
    done = 0
    while done < n_events:
        m = min(chunk, n_events - done)
        p1, p2 = fill(True, m)
        d1, d2 = fill(False, m)
        isd = torch.rand(m, generator=g, device=dev) < delayed_frac
        k = torch.arange(done, done + m, device=dev)
        slot = k + k // events_per_ms + 1
        out[2 * slot] = _to_i32(torch, torch.where(isd, d1, p1))
        out[2 * slot + 1] = _to_i32(torch, torch.where(isd, d2, p2))
        done += m
    t = torch.arange(ntags, device=dev)
    tag = 0x80000000 | t
    tslot = t * (events_per_ms + 1)
    out[2 * tslot] = _to_i32(torch, 0x40000000 | (tag & 0xFFFF))
    out[2 * tslot + 1] = _to_i32(torch, 0xC0000000 | ((tag >> 16) & 0xFFFF))
    return out
