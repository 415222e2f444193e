"""The eigensolver's distributed round-robin schedule (CPU only).

k_jacobi (am1-rs_b200/csrc/k_linalg.cu) spreads the columns of one matrix over a cluster of 1..16
CTAs and moves one column per neighbour per step.  This is a line-by-line Python model of the
kernel's ring bookkeeping (heads, edge CTAs, landing buffers); it checks that every column pair
meets exactly once per sweep, that buffer indices stay in range, and that no column is lost.
"""


def simulate(n, C):
    npad = ((max(n, 2) + 2*C - 1) // (2*C)) * (2*C)
    m = npad // 2; q = m // C
    if C > 1 and q < 2: return None
    nbuf = 2*q + 2; LT_, LB_ = 2*q, 2*q+1
    # per CTA state
    cta = []
    for c in range(C):
        colid = [None]*nbuf
        for b in range(2*q):
            colid[b] = c*q + b if b < q else m + c*q + (b - q)
        T = list(range(q)); B = list(range(q, 2*q))
        if C > 1 and c == 0:
            fixed = T[0]; T = T[1:] + [fixed]
        cta.append(dict(colid=colid, T=T, B=B, ht=0, hb=0))
    L1 = 2*q - 1
    def top_buf(c, k, s):
        st = cta[c]; T, B = st['T'], st['B']
        if C == 1:
            if k == 0: return T[0]
            r = k - 1; src = (r - s) % L1
            return T[1+src] if src < q-1 else B[q-1-(src-(q-1))]
        if c == 0 and k == 0: return T[q-1]
        qt = q-1 if c == 0 else q
        kk = k-1 if c == 0 else k
        return T[(st['ht'] + kk) % qt]
    def bot_buf(c, k, s):
        st = cta[c]; T, B = st['T'], st['B']
        if C == 1:
            r = L1 - 1 - k; src = (r - s) % L1
            return T[1+src] if src < q-1 else B[q-1-(src-(q-1))]
        return B[(st['hb'] + k) % q]
    for sweep in range(2):
        met = set()
        for s in range(npad - 1):
            # rotations
            for c in range(C):
                used = set()
                for k in range(q):
                    bp, bq = top_buf(c, k, s), bot_buf(c, k, s)
                    assert 0 <= bp < 2*q and 0 <= bq < 2*q, (bp, bq)
                    assert bp not in used and bq not in used and bp != bq
                    used |= {bp, bq}
                    a, b2 = cta[c]['colid'][bp], cta[c]['colid'][bq]
                    pr = (min(a, b2), max(a, b2))
                    assert pr not in met, ("pair twice", pr, s)
                    met.add(pr)
                assert len(used) == 2*q
            if C == 1: continue
            # exchange (content = colid)
            LT = [top_buf(c, q-1, s) for c in range(C)]
            LB = [bot_buf(c, 0, s) for c in range(C)]
            for c in range(C):
                if c < C-1: cta[c+1]['colid'][LT_] = cta[c]['colid'][LT[c]]
                if c > 0: cta[c-1]['colid'][LB_] = cta[c]['colid'][LB[c]]
            for c in range(C):
                st = cta[c]; qt = q-1 if c == 0 else q
                ht, hb = st['ht'], st['hb']
                nht, nhb = (ht - 1 + qt) % qt, (hb + 1) % q
                ct = cb = -1
                if c == 0:
                    cb = LT[c]; st['T'][nht] = LB[c]; st['B'][hb] = LT[c]
                elif c == C-1:
                    ct = LB[c]; st['T'][nht] = LB[c]; st['B'][hb] = LT[c]
                else:
                    ct = LT[c]; cb = LB[c]
                if ct >= 0: st['colid'][ct] = st['colid'][LT_]
                if cb >= 0: st['colid'][cb] = st['colid'][LB_]
                st['ht'], st['hb'] = nht, nhb
        want = npad*(npad-1)//2
        assert len(met) == want, (n, C, len(met), want)
    # all columns still present exactly once
    cols = sorted(cta[c]['colid'][b] for c in range(C) for b in
                  ([cta[c]['T'][i] for i in range(len(cta[c]['T']))] + cta[c]['B']))
    assert cols == list(range(npad)), cols
    return npad

def test_every_pair_meets_once_per_sweep():
    for C in (1, 2, 4, 8, 16):
        for n in list(range(1, 70)) + [111, 112, 160, 192, 224, 242, 320, 384, 448]:
            simulate(n, C)
