"""CPU test: multi-limb constants written into the CUDA sources match the
values computed from p (a wrong limb would corrupt results silently)."""
import os
import re

P = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "icp-gpu_b200", "csrc")


def limbs32(x, n=12):
    return [(x >> (32 * i)) & 0xFFFFFFFF for i in range(n)]


def arrays(text):
    """name -> list of ints for `... NAME[12] = {...}` (32-bit limb arrays)."""
    out = {}
    for m in re.finditer(r"(\w+)\[12\]\s*=\s*\{([^}]*)\}", text):
        items = [v.strip() for v in m.group(2).split(",") if v.strip()]
        if not all(re.fullmatch(r"0x[0-9a-fA-F]+[uUlL]*", v) for v in items):
            continue
        vals = [int(re.sub(r"[uUlL]+$", "", v), 16) for v in items]
        out.setdefault(m.group(1), []).append(vals)
    return out


def test_verify_vm_multiples_of_p():
    with open(os.path.join(CSRC, "verify_vm.cu")) as f:
        a = arrays(f.read())
    assert a["P4"][0] == limbs32(4 * P)
    assert a["P2"][0] == limbs32(2 * P)


def test_vm_offsets_and_exponents():
    with open(os.path.join(CSRC, "vm.cuh")) as f:
        a = arrays(f.read())
    assert limbs32(8 * P) in a["e"]
    assert limbs32(P - 2) in a["e"]


def test_g1_constants():
    with open(os.path.join(CSRC, "g1.cuh")) as f:
        text = f.read()
    a = arrays(text)
    assert a["h"][0] == limbs32((P - 1) // 2)
    beta = 0x5f19672fdf76ce51ba69c6076a0f77eaddb3a93be6f89688de17d813620a00022e01fffffffefffe
    m = re.search(r"bv\[6\] = \{([^}]*)\}", text)
    vals = [int(v.strip().rstrip("ULL"), 16) for v in m.group(1).split(",")]
    mont = beta * (1 << 384) % P
    assert vals == [(mont >> (64 * i)) & (2**64 - 1) for i in range(6)]
    assert pow(beta, 3, P) == 1 and beta != 1


def test_fp_header_constants():
    with open(os.path.join(CSRC, "fp.cuh")) as f:
        text = f.read()
    ps = [int(x, 16) for x in re.findall(r"#define BLS_P\d+ (0x[0-9a-f]+)u", text)]
    assert ps == limbs32(P)
    assert int(re.search(r"#define BLS_NINV (0x[0-9a-f]+)u", text).group(1), 16) == (-pow(P, -1, 2**32)) % 2**32
