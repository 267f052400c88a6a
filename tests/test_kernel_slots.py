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
    kp = (17 + 1) * 64
    total = (slot_u4 + k_u4 + xch_u4) * 16 + kp + 4 * v * 4 + 16 * v + 16
    assert total <= 227 * 1024
    src = open(os.path.join(CSRC, "verify_w.cu")).read()
    for name in ("kItemSlots = kCOff + 12", "kSlotU4 = kItemSlots * 6 * kV", "kXchU4 = 6 * 2 * 7 * kV"):
        assert name in src
