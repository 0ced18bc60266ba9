"""Shared-memory bank model of the four-step line walk (sj_lines.cuh, fs_forward).

The two-pass kernels (sj_kernels.cuh) choose their tile pitches with this model: a column strip of
256-point lines uses pitch tc + 2 and row blocks of 256- and 512-point lines use pitch w + 8 and
w + 16.  For 128- and 256-point lines (G = 4, 8) the stage-2 rounds pair lines whose exchange slots lie
16 banks apart (fs_slot / FsTasks in sj_lines.cuh).  The tests recount the wavefronts of one warp's
forward four-step (Makhoul gather, exchange stores and loads, post-rotation stores) and check that
the chosen pitches and the paired rounds need fewer than pitch + 4 and rounds of consecutive tasks.  A wavefront count of one warp access is the largest number of
distinct 32-bit words that fall into one of the 32 banks.
"""


def wavefronts(addrs):
    banks = {}
    for a in addrs:
        if a is not None:
            banks.setdefault(a % 32, set()).add(a)
    return max((len(s) for s in banks.values()), default=0)


def makhoul_src(n, big_n):
    return 2 * n if n < big_n // 2 else 2 * big_n - 1 - 2 * n


def bitrev(b, g):
    bits = g.bit_length() - 1
    return int(format(b, f"0{bits}b")[::-1], 2) if bits else 0


def fs_slot(g, j, rows):
    half = 32 // g // 2
    return (j >> 1) + half * (j & 1) if (g in (4, 8) and not rows) else j


def rounds_of(g, rows, paired):
    """Stage-2 (line, column) task of each lane, per round."""
    lpw = 32 // g
    if g in (4, 8) and paired:
        return [[((r + lpw // 2 * (l // 15)) if rows else (2 * r + l // 15), 1 + l % 15) if l < 30 else None
                 for l in range(32)] for r in range(lpw // 2)]
    ntask = lpw * 15
    return [[(t // 15, 1 + t % 15) if t < ntask else None for t in range(r, r + 32)] for r in range(0, ntask, 32)]


def four_step_wavefronts(g, pitch, rows, paired=True):
    """Wavefronts of one warp's fs_forward for G = g (line length 32 g); rows: lines are tile rows
    (element stride 1, line stride pitch), else tile columns (element stride pitch, line stride 1).
    paired: the kernel's stage-2 rounds and exchange slots; else consecutive tasks, slot = line."""
    n = 32 * g
    lpw = 32 // g
    xp = g + 1                                       # FourStepSizes<G>::PITCH
    line_len = {4: 84, 8: 168, 16: 304}.get(g, 17 * xp)   # FourStepSizes<G>::LINE
    plane = lpw * line_len
    es = 1 if rows else pitch
    base = (lambda j: j * pitch) if rows else (lambda j: j)
    slot = (lambda j: fs_slot(g, j, rows)) if paired else (lambda j: j)
    total = 0
    for a in range(32):                               # stage-1 Makhoul gather
        total += wavefronts([base(l // g) + makhoul_src(g * a + l % g, n) * es for l in range(32)])
    for c in range(1, 16):                            # twiddled stage-1 outputs into the exchange
        for pl in (0, 1):
            total += wavefronts([pl * plane + slot(l // g) * line_len + l % g + c * xp for l in range(32)])
    for col in (0, 16):                               # post rotation of columns 0 and 16
        for side in (0, 1):
            addrs = []
            for l in range(32):
                d = bitrev(l % g, g)
                k = 32 * d + col
                ok = d <= g // 2 if col == 0 else d < g // 2
                if not ok or (side == 1 and (k == 0 or 2 * k == n)):
                    addrs.append(None)
                else:
                    addrs.append(base(l // g) + (k if side == 0 else n - k) * es)
            total += wavefronts(addrs)
    for tasks in rounds_of(g, rows, paired):          # stage 2: tasks (line, column c = 1..15)
        for q in range(g):
            for pl in (0, 1):
                total += wavefronts([None if t is None else pl * plane + slot(t[0]) * line_len + t[1] * xp + q
                                     for t in tasks])
        for dd in range(g):
            for side in (0, 1):
                total += wavefronts([None if t is None else
                                     base(t[0]) + ((t[1] + 32 * dd) if side == 0 else n - t[1] - 32 * dd) * es
                                     for t in tasks])
    return total


def test_strip_pitch_of_256_point_columns():
    tc = 32
    assert four_step_wavefronts(8, tc + 2, rows=False) < 0.85 * four_step_wavefronts(8, tc + 4, rows=False)


def test_row_block_pitches_of_256_and_512_point_rows():
    assert four_step_wavefronts(8, 256 + 8, rows=True) < 0.8 * four_step_wavefronts(8, 256 + 4, rows=True)
    assert four_step_wavefronts(16, 512 + 16, rows=True) < 0.9 * four_step_wavefronts(16, 512 + 4, rows=True)


def test_paired_stage2_rounds_of_128_and_256_point_lines():
    for rows, pitch in ((True, 256 + 8), (False, 32 + 2), (False, 32 + 4)):
        assert four_step_wavefronts(8, pitch, rows) < 0.9 * four_step_wavefronts(8, pitch, rows, paired=False)
    for rows, pitch in ((True, 128 + 4), (False, 64 + 4)):
        assert four_step_wavefronts(4, pitch, rows) < 0.8 * four_step_wavefronts(4, pitch, rows, paired=False)


def test_even_pitch_of_512_point_strips_costs_no_more_than_the_odd_one():
    # 32-column strips of 512-point lines use pitch 34 instead of 33 so that they load asynchronously
    assert four_step_wavefronts(16, 34, rows=False) <= four_step_wavefronts(16, 33, rows=False)


def test_odd_pitch_of_1024_point_strips():
    # 1024-point column strips keep the odd pitch tc + 1: with 32 lanes on one line, an even pitch
    # puts pairs of gather lanes in one bank (tc + 2 counts about 22% more wavefronts)
    for tc in (8, 16):
        odd, even = four_step_wavefronts(32, tc + 1, rows=False), four_step_wavefronts(32, tc + 2, rows=False)
        assert even > 1.2 * odd


def g32_post_store_wavefronts(es, swapped):
    """Stage-2 post-rotation stores of a 1024-point line (G = 32): lane l < 30 owns column
    c = 1 + l // 2 and the half h = l % 2 (d = 2 m + h); at step m it stores y[k] and y[N - k],
    k = c + 32 d.  swapped: lanes with h = 1 store y[N - k] first (fs_forward)."""
    n, total = 1024, 0
    for m in range(16):
        first, second = [], []
        for l in range(32):
            if l >= 30:
                first.append(None)
                second.append(None)
                continue
            c, h = 1 + l // 2, l % 2
            k = c + 32 * (2 * m + h)
            a, b = (n - k, k) if (swapped and h) else (k, n - k)
            first.append(a * es)
            second.append(b * es)
        total += wavefronts(first) + wavefronts(second)
    return total


def test_g32_post_stores_are_bank_disjoint_after_the_swap():
    # rows (es = 1) and the odd pitches of 1024-point column strips (tc + 1 = 9, 17)
    for es in (1, 9, 17):
        assert g32_post_store_wavefronts(es, swapped=True) == 32          # one wavefront per store
        assert g32_post_store_wavefronts(es, swapped=False) == 64         # lanes (c, 0), (c, 1) collide


def test_paired_row_gather_has_no_conflicts():
    """Row lines read Makhoul's v[n] = x[2n], v[N-1-n] = x[2n+1] as 64-bit pairs: one 64-bit access
    per lane (two wavefronts for 32 lanes, the minimum) instead of two scalar stride-2 accesses of
    two wavefronts each."""
    for g, pitch in ((4, 128 + 4), (8, 256 + 8), (16, 512 + 16), (32, 1024 + 4)):   # the row-block pitches
        n = 32 * g
        pair_words = []
        for a in range(16):
            words = []
            for l in range(32):
                j, b = l // g, l % g
                words += [j * pitch + 2 * (g * a + b), j * pitch + 2 * (g * a + b) + 1]
            # a 64-bit warp access is serviced per half warp
            pair_words.append(wavefronts(words[:32]) + wavefronts(words[32:]))
        scalar = [wavefronts([(l // g) * pitch + makhoul_src(g * a + l % g, n) for l in range(32)])
                  for a in range(32)]
        # half the instructions always and never more wavefronts; conflict-free for 512- and
        # 1024-point rows (one line per half warp).  128- and 256-point rows, several lines per half
        # warp at the pitches the scalar model chose (132, 264), keep the scalar gather's count.
        assert sum(pair_words) <= sum(scalar), g
        if g >= 16:
            assert sum(pair_words) == 32 and sum(scalar) == 64, (g, sum(pair_words), sum(scalar))


def test_transposed_512_point_strips():
    """512-point column strips (32 wide) are staged transposed at pitch 529: the column lines then
    walk as rows, which the model counts cheaper than the 34-pitch column walk, and the transposing
    scalar stores of the staging (a warp: 4 rows x 8 float4 groups) are conflict-free; so are those
    of the 1024-point strips, 16 wide at pitch 1026 and 8 wide at 1028 (not at each other's)."""
    assert four_step_wavefronts(16, 529, rows=True) < 0.9 * four_step_wavefronts(16, 34, rows=False)
    for pitch, tc in ((529, 32), (1028, 8), (1026, 16)):
        q = tc // 4
        for j in range(4):
            assert wavefronts([(4 * (l % q) + j) * pitch + l // q for l in range(32)]) == 1
    for pitch, tc in ((1028, 16), (1026, 8)):
        q = tc // 4
        assert max(wavefronts([(4 * (l % q) + j) * pitch + l // q for l in range(32)]) for j in range(4)) == 2


def test_padded_arrays_make_narrow_tile_columns_conflict_free():
    """Whole-array tiles of 8- and 16-column arrays (pitch w + 4): h * (w + 4) is a multiple of 32
    floats, so a warp's 32 register-line column walks over 4 or 2 arrays share banks; padding the
    arrays to 8 / 16 (mod 32) floats apart (tile_array_pitch in sj_kernels.cuh) removes it."""
    def tile_array_pitch(h, w, p):
        if w == 8 and h <= 128:
            return h * p + (40 - (h * p) % 32) % 32
        if w == 16 and h <= 64:
            return h * p + (48 - (h * p) % 32) % 32
        return h * p

    for h, w in [(16, 8), (32, 8), (64, 8), (128, 8), (8, 16), (16, 16), (32, 16), (64, 16), (8, 8)]:
        p = w + 4
        ap = tile_array_pitch(h, w, p)
        assert ap % 4 == 0                                    # rows stay 16-byte aligned
        plain = sum(wavefronts([(l // w) * h * p + i * p + l % w for l in range(32)]) for i in range(h))
        padded = sum(wavefronts([(l // w) * ap + i * p + l % w for l in range(32)]) for i in range(h))
        assert padded == h, (h, w)
        assert plain == h * 32 // w, (h, w)                  # 4-way (w = 8), 2-way (w = 16) before


def test_tile_pitches_of_four_step_axes_beside_register_lines():
    """Whole-array tiles whose one axis runs the four-step and the other register lines take the
    two-pass kernels' pitches for the four-step axis (tile_pitch in sj_kernels.cuh): 256-point
    columns w + 2, 256- and 512-point rows w + 8 and w + 16.  Where both axes run the four-step
    (256 x 128, 128 x 256) w + 4 is as good or better for the two walks together."""
    for w in (8, 16, 32, 64):
        assert four_step_wavefronts(8, w + 2, rows=False) < 0.75 * four_step_wavefronts(8, w + 4, rows=False)
    assert four_step_wavefronts(8, 264, rows=True) < 0.7 * four_step_wavefronts(8, 260, rows=True)
    assert four_step_wavefronts(16, 528, rows=True) < 0.9 * four_step_wavefronts(16, 516, rows=True)
    both = lambda p, gc, gr: four_step_wavefronts(gc, p, rows=False) + four_step_wavefronts(gr, p, rows=True)
    assert both(132, 8, 4) < both(130, 8, 4)          # 256 x 128
    assert both(260, 4, 8) <= both(264, 4, 8)         # 128 x 256
