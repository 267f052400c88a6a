"""Static check of the six-lane kernels' shared-memory slot plan, on the CPU.

Both Fp2-lane kernels (verify_fp2.cu: five items per block; verify_w.cu: 32
items per block, item-interleaved) resolve every slot reference of a program
as base + index, with the bases of the op: D, A, B the op's Fp12 groups, C the
line / point area, K the block-shared constants, T the inverse's temporaries.
Every reference of every program that the op sequences run must land inside
the per-item slot area (reads may also name the constants), and every write
must land in the per-item area, never in the constants: the kernels compute
shared-memory addresses from these indices without further checks."""
import os
import re
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "icp-gpu_b200", "csrc"))
import gen_fp2ops as G  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "icp-gpu_b200", "csrc")


def _kernel_constants():
    inc = open(os.path.join(CSRC, "fp2ops.inc")).read()
    k_slots = int(re.search(r"constexpr int kKSlotCount = (\d+);", inc).group(1))
    groups = int(re.search(r"constexpr int kGroupsUsed = (\d+);", inc).group(1))
    t_group = int(re.search(r"constexpr int kTGroup = (\d+);", inc).group(1))
    return k_slots, groups, t_group


def _refs(o):
    reads = []
    for t in o.terms:
        reads.append(t.x)
        if t.y is not None:
            reads.append(t.y)
    reads += [r for _, r in o.lins]
    return reads, o.dst


def test_every_slot_reference_is_inside_the_item_area():
    k_slots, groups, t_group = _kernel_constants()
    c_off = 6 * groups
    item_slots = c_off + 12                       # groups, then the 12-slot C area
    lo, hi = k_slots, k_slots + item_slots        # per-item slots (absolute)
    assert hi <= 256                              # slot indices travel in one byte
    progs = {name: outs for name, outs, _ in G.build()}
    names = [n for n, _, _ in G.PROGRAMS]
    checked = 0
    for normalised in (False, True):
        for op in G.driver_sequence(normalised):
            code, d, a, b, _ = op
            code &= ~G.COND_ML
            if code >= len(names):
                assert code in (G.OP_LOAD_CORR, G.OP_MILLER_DONE, G.OP_LOAD_LINES)
                if code == G.OP_MILLER_DONE:
                    assert 0 <= d < groups
                continue
            assert max(d, a, b) < groups
            bases = {G.B_D: lo + 6 * d, G.B_A: lo + 6 * a, G.B_B: lo + 6 * b, G.B_C: lo + c_off, G.B_K: 0,
                     G.B_T: lo + 6 * t_group}
            for o in progs[names[code]]:
                if o is None:
                    continue
                reads, dst = _refs(o)
                for r in reads:
                    s = bases[r >> 4] + (r & 15)
                    if (r >> 4) == G.B_K:
                        assert 0 <= s < k_slots
                    else:
                        assert lo <= s < hi, (names[code], hex(r), s)
                    checked += 1
                s = bases[dst >> 4] + (dst & 15)
                assert (dst >> 4) != G.B_K and lo <= s < hi, (names[code], hex(dst), s)
                checked += 1
    assert checked > 10000


def test_wide_kernel_layout_fits_one_block_per_sm():
    """The 32-item kernel's shared memory (computed as verify_w.cu does) fits
    the 227 KB a block may use, and its per-item slot area matches the plan."""
    k_slots, groups, _ = _kernel_constants()
    item_slots = 6 * groups + 12
    v = 32
    slot_u4 = item_slots * 6 * v
    k_u4 = k_slots * 6
    xch_u4 = 6 * 2 * 7 * v
    qp_u4 = 128 * 4
    kp = (17 + 1) * 64
    total = (slot_u4 + k_u4 + xch_u4 + qp_u4) * 16 + kp + 4 * v * 4 + 16 * v + 16
    assert total <= 227 * 1024
    src = open(os.path.join(CSRC, "verify_w.cu")).read()
    for name in ("kItemSlots = kCOff + 12", "kSlotU4 = kItemSlots * 6 * kV", "kXchU4 = 6 * 2 * 7 * kV",
                 "kQpU4 = 128 * 4"):
        assert name in src


def test_every_program_writes_no_slot_it_reads():
    """The generator sends every result that would overwrite an operand to a
    group whose value is dead; the final exponentiation holds at most six
    live values, so with seven groups one is always free.  No program of
    either sequence then writes a slot that one of its outputs reads, which
    the 32-item kernel relies on when it stores a program's outputs without
    a block barrier after the reads; each op's word carries the flag."""
    n_prog = len(G.PROGRAMS)
    for normalised in (False, True):
        logical = G.logical_sequence(normalised)
        live = G.live_after(logical)
        busiest = 0
        progs = 0
        for i, op in enumerate(G.driver_sequence(normalised)):
            if (op[0] & ~G.COND_ML) >= n_prog:
                assert not G.encode_op(op) & G.NO_WAR
                continue
            rd, wr = G.op_slots(op)
            assert not (rd & wr), op
            assert G.encode_op(op) & G.NO_WAR
            code, d, a, b, _ = logical[i]
            rb, _ = G.program_io(code & ~G.COND_ML)
            srcs = ({a} if G.B_A in rb else set()) | ({b} if G.B_B in rb else set())
            busiest = max(busiest, len((live[i] - {d}) | srcs))
            progs += 1
        assert progs > 640 and busiest < G.PHYS_GROUPS


def test_inverse_temporaries_hold_no_live_value():
    """The inverse's temporaries (base T, from group kTGroup) overwrite only
    groups whose values are dead: walking each sequence backwards from the
    final read of Gt, no group that a later op still reads lies under a slot
    an inverse program writes (ops that run only when the Miller value is
    wanted count as readers but never as writers)."""
    n_prog = len(G.PROGRAMS)
    for normalised in (False, True):
        seq = G.driver_sequence(normalised)
        live = {G.gt_group(normalised)}
        checked = 0
        for op in reversed(seq):
            code, d, a, b, _ = op
            c = code & ~G.COND_ML
            if c == G.OP_MILLER_DONE:
                live.add(d)
                continue
            if c >= n_prog:
                continue
            rb, wb = G.program_io(c)
            if G.B_T in wb:
                t_groups = {G.T_GROUP + (o.dst & 15) // 6 for o in G.PROGRAMS[c][1]() if o is not None
                            and (o.dst >> 4) == G.B_T}
                assert not (t_groups & live), (G.PROGRAMS[c][0], t_groups, live)
                checked += 1
            if G.B_D in wb and not code & G.COND_ML:
                live.discard(d)
            if G.B_A in rb:
                live.add(a)
            if G.B_B in rb:
                live.add(b)
        assert checked == 7
