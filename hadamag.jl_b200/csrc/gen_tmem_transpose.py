"""Generate tmem_transpose.cuh: lane <-> register exchanges of the warp engine through
tensor memory (TMEM), for the exact-SRE pass-1 rows and pass-2 tiles.

    python hadamag.jl_b200/csrc/gen_tmem_transpose.py

A warp holds 32 complex values per lane (FP64: 4 32-bit words each, FP32: 2).  An
exchange moves some of the element-index bits held by the lane number into the register
index, and register bits into the lane number, through rounds of a TMEM store and a TMEM
load with different access shapes.  Per 16-lane half h of the warp's 32 TMEM lanes, the
shapes place thread t's register rho at (lane, column):

  32x32b   lane t,                           column rho
  16x256b  lane 16h + 8 v + (t >> 2),         column 8 k + 2 (t & 3) + u    (rho = 4k + 2v + u)
  16x64b   lane 16h + 8 (t & 1) + (t >> 2),   column 2 k + ((t >> 1) & 1)  (rho = k)

(measured on B200 with tcgen05.st / tcgen05.ld of every shape).  A round stores with one
shape and loads with another:

  DOWN2  st 16x256b, ld 32x32b: new lane bits (t0..t4) = (t2, t3, t4, v, h); the
         old lane bits t0, t1 become register bits
  DOWN1  st 16x64b,  ld 32x32b: new lane bits = (t2, t3, t4, t0, h); old t1 -> register
  UP2    st 32x32b,  ld 16x256b: new lane bits = (c1, c2, t0, t1, t2) (c = column bits);
         old t3, t4 -> register
  UP1    st 32x32b,  ld 16x64b: new lane bits = (t3, c0, t0, t1, t2); old t4 -> register

The register bits that go to the lane number (h, v, or column bits) are chosen per round;
the others keep their order.  Every operand index is a compile-time literal, so the
generated code only renames registers around the TMEM instructions.
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "tmem_transpose.cuh")


class Layout:
    """Bit labels of the lane number (tb[0] = lane bit 0) and of the flat word-register
    index (rb[0] = register bit 0)."""

    def __init__(self, tb, rb):
        self.tb = list(tb)
        self.rb = list(rb)

    def reg_index(self, labels):
        """register index of the word with the given label values (dict label -> bit)"""
        return sum(labels[b] << i for i, b in enumerate(self.rb))


def src_order(lay, chosen_positions, m):
    """Source index bit -> label: `chosen_positions` maps source bit positions to the labels
    chosen for them; the other current register labels fill the remaining positions in
    their current order."""
    rest = [b for b in lay.rb if b not in chosen_positions.values()]
    out = []
    it = iter(rest)
    for pos in range(m):
        out.append(chosen_positions[pos] if pos in chosen_positions else next(it))
    return out


def round_down2(lay, h, v, m):
    # source index: bit0 = u, bit1 = v, bits 2 .. m-2 = k, bit m-1 = h
    src = src_order(lay, {m - 1: h, 1: v}, m)
    t = lay.tb
    new_tb = [t[2], t[3], t[4], v, h]
    # dest column = 8k + 2 (t1 t0) + u: bit0 = u, bit1 = t0, bit2 = t1, bits 3.. = k
    new_rb = [src[0], t[0], t[1]] + src[2:m - 1]
    return src, Layout(new_tb, new_rb)


def round_down1(lay, h, m):
    # source index: bits 0 .. m-2 = k, bit m-1 = h
    src = src_order(lay, {m - 1: h}, m)
    t = lay.tb
    new_tb = [t[2], t[3], t[4], t[0], h]
    # dest column = 2k + t1
    new_rb = [t[1]] + src[0:m - 1]
    return src, Layout(new_tb, new_rb)


def round_up2(lay, c2, c1, m):
    # source index = column: bit1 = c1, bit2 = c2
    src = src_order(lay, {1: c1, 2: c2}, m)
    t = lay.tb
    new_tb = [src[1], src[2], t[0], t[1], t[2]]
    # dest register = (NW/2) h + 4k + 2v + u: u = col0, v = t3, k = col bits 3.., h = t4
    new_rb = [src[0], t[3]] + src[3:m] + [t[4]]
    return src, Layout(new_tb, new_rb)


def round_up1(lay, c0, m):
    # source index = column: bit0 = c0
    src = src_order(lay, {0: c0}, m)
    t = lay.tb
    new_tb = [t[3], src[0], t[0], t[1], t[2]]
    # dest register = (NW/2) h + k, k = col >> 1, h = t4
    new_rb = src[1:m] + [t[4]]
    return src, Layout(new_tb, new_rb)


def operand_list(prev, src, nw):
    """operand j of the store = the current register holding the word whose labels give
    source index j"""
    ops = []
    for j in range(nw):
        labels = {b: (j >> i) & 1 for i, b in enumerate(src)}
        ops.append(prev.reg_index(labels))
    return ops


def emit_st(kind, base_expr, regs, arr):
    """tcgen05.st of the given registers (two 16-lane halves for the 16x shapes)"""
    lines = []
    nw = len(regs)
    if kind == "32x32b":
        ops = ",".join(f"%{i + 1}" for i in range(nw))
        args = ", ".join(f'"r"({arr}[{r}])' for r in regs)
        lines.append(f'  asm volatile("tcgen05.st.sync.aligned.32x32b.x{nw}.b32 [%0], {{{ops}}};" '
                     f'::"r"({base_expr}), {args} : "memory");')
        return lines
    half = nw // 2
    reps = half // 4 if kind == "16x256b" else half
    for h in range(2):
        part = regs[h * half:(h + 1) * half]
        ops = ",".join(f"%{i + 1}" for i in range(half))
        args = ", ".join(f'"r"({arr}[{r}])' for r in part)
        lines.append(f'  asm volatile("tcgen05.st.sync.aligned.{kind}.x{reps}.b32 [%0], {{{ops}}};" '
                     f'::"r"({base_expr} + {16 * h}u * 65536u), {args} : "memory");')
    return lines


def emit_ld(kind, base_expr, nw, arr):
    lines = []
    if kind == "32x32b":
        ops = ",".join(f"%{i}" for i in range(nw))
        outs = ", ".join(f'"=r"({arr}[{i}])' for i in range(nw))
        lines.append(f'  asm volatile("tcgen05.ld.sync.aligned.32x32b.x{nw}.b32 {{{ops}}}, [%{nw}];" '
                     f': {outs} : "r"({base_expr}) : "memory");')
        return lines
    half = nw // 2
    reps = half // 4 if kind == "16x256b" else half
    for h in range(2):
        ops = ",".join(f"%{i}" for i in range(half))
        outs = ", ".join(f'"=r"({arr}[{h * half + i}])' for i in range(half))
        lines.append(f'  asm volatile("tcgen05.ld.sync.aligned.{kind}.x{reps}.b32 {{{ops}}}, [%{half}];" '
                     f': {outs} : "r"({base_expr} + {16 * h}u * 65536u) : "memory");')
    return lines


SHAPES = {"DOWN2": ("16x256b", "32x32b"), "DOWN1": ("16x64b", "32x32b"),
          "UP2": ("32x32b", "16x256b"), "UP1": ("32x32b", "16x64b")}


def gen_function(name, fp64, lane_labels, reg_elem_labels, rounds, canon):
    """lane_labels: element bits on lane bits 0..4; reg_elem_labels: element bits of the
    element register index i (bit 0 first); rounds: list of (kind, chosen labels); canon:
    element labels of the output register index, bit 0 first."""
    wbits = ["q0", "q1"] if fp64 else ["q0"]
    nw = 32 * (4 if fp64 else 2)
    m = nw.bit_length() - 1
    lay = Layout(lane_labels, wbits + reg_elem_labels)
    body = []
    body.append(f"  uint32_t a[{nw}], b[{nw}];")
    # pack: word w of element i at register w + (4 or 2) i of the initial layout
    for i in range(32):
        if fp64:
            idx = lambda w: w + 4 * i  # noqa: E731
            body.append(f"  a[{idx(0)}] = __double2loint(v[{i}].x); a[{idx(1)}] = __double2hiint(v[{i}].x); "
                        f"a[{idx(2)}] = __double2loint(v[{i}].y); a[{idx(3)}] = __double2hiint(v[{i}].y);")
        else:
            body.append(f"  a[{2 * i}] = __float_as_uint(v[{i}].x); a[{2 * i + 1}] = __float_as_uint(v[{i}].y);")
    cur, nxt = "a", "b"
    for kind, chosen in rounds:
        if kind == "DOWN2":
            src, new = round_down2(lay, chosen[0], chosen[1], m)
        elif kind == "DOWN1":
            src, new = round_down1(lay, chosen[0], m)
        elif kind == "UP2":
            src, new = round_up2(lay, chosen[0], chosen[1], m)
        else:
            src, new = round_up1(lay, chosen[0], m)
        st_shape, ld_shape = SHAPES[kind]
        ops = operand_list(lay, src, nw)
        body += emit_st(st_shape, "taddr", ops, cur)
        body.append('  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");')
        body += emit_ld(ld_shape, "taddr", nw, nxt)
        body.append('  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");')
        lay = new
        cur, nxt = nxt, cur
    # unpack: output element j (bits of `canon`) word w
    for b in canon:
        assert b in lay.rb, (name, b, lay.rb)
    for j in range(32):
        labels = {b: (j >> i) & 1 for i, b in enumerate(canon)}

        def reg(wv):
            lab = dict(labels)
            lab["q0"] = wv & 1
            if fp64:
                lab["q1"] = wv >> 1
            return lay.reg_index(lab)
        if fp64:
            body.append(f"  v[{j}].x = __hiloint2double({cur}[{reg(1)}], {cur}[{reg(0)}]); "
                        f"v[{j}].y = __hiloint2double({cur}[{reg(3)}], {cur}[{reg(2)}]);")
        else:
            body.append(f"  v[{j}].x = __uint_as_float({cur}[{reg(0)}]); v[{j}].y = __uint_as_float({cur}[{reg(1)}]);")
    V = "double2" if fp64 else "float2"
    doc = (f"// lanes {lay.tb} after the exchange; output register j holds element bits "
           f"{canon} (bit 0 first)")
    return (f"{doc}\n__device__ __forceinline__ void {name}({V} (&v)[32], uint32_t taddr) {{\n"
            + "\n".join(body) + "\n}\n")


def main():
    E = [f"e{i}" for i in range(10)]
    funcs = []
    for fp64 in (True, False):
        sfx = "f64" if fp64 else "f32"
        # pass 1: row of 1024 elements, lanes e0..e4, registers e5..e9; all five lane bits
        # go to registers (DOWN1, DOWN2, DOWN2), output registers = e0..e4
        funcs.append(gen_function(f"tmem_xchg_row_{sfx}", fp64, E[0:5], E[5:10],
                                  [("DOWN1", ["e5"]), ("DOWN2", ["e6", "e7"]), ("DOWN2", ["e8", "e9"])],
                                  E[0:5]))
        # pass 2: tile of 2^HI rows x C = 2^LOGC positions, element e = row C + c; lanes hold
        # the C bits and row bits r0 .. r(4 - LOGC); those row bits go to registers and sit at
        # output register bits 0 .. 4 - LOGC, followed by the other register bits
        for logc in range(0, 5):
            hi = 10 - logc
            lab = [f"c{j}" for j in range(logc)] + [f"r{j}" for j in range(hi)]
            lanes, regs = lab[0:5], lab[5:10]
            rows_in_lanes = [b for b in lanes if b.startswith("r")]
            k = len(rows_in_lanes)
            if k == 5:
                rounds = [("DOWN1", [regs[0]]), ("DOWN2", [regs[1], regs[2]]), ("DOWN2", [regs[3], regs[4]])]
            elif k == 4:
                rounds = [("UP2", [regs[0], regs[1]]), ("UP2", [regs[2], regs[3]])]
            elif k == 3:
                rounds = [("UP2", [regs[0], regs[1]]), ("UP1", [regs[2]])]
            elif k == 2:
                rounds = [("UP2", [regs[0], regs[1]])]
            else:
                rounds = [("UP1", [regs[0]])]
            # output: the moved row bits first, then the register bits that stayed
            stay = [b for b in regs if b not in sum((r[1] for r in rounds), [])]
            canon = rows_in_lanes + stay
            funcs.append(gen_function(f"tmem_xchg_tile{hi}_{sfx}", fp64, lanes, regs, rounds, canon))
    hdr = ('// tmem_transpose.cuh -- GENERATED by gen_tmem_transpose.py (do not edit): lane <-> register\n'
           '// exchanges of the warp engine through tensor memory.  `taddr` is the TMEM address of\n'
           '// this warp\'s 32 lanes (column base of its allocation); the exchange uses 128 (FP64)\n'
           '// or 64 (FP32) columns.\n'
           '//   tmem_xchg_row_*: a 1024-element pass-1 row, lanes e0..e4 / registers e5..e9 in,\n'
           '//     registers e0..e4 out (register j = element bits of j in that order).\n'
           '//   tmem_xchg_tile<HI>_*: a pass-2 tile of 2^HI rows x 2^(10-HI) positions loaded as\n'
           '//     element 32 i + lane; out: the row bits that sat on lanes are register bits\n'
           '//     0 .. (HI - 6), lowest row bit first.\n'
           '#pragma once\n#include <cuda_runtime.h>\n#include <stdint.h>\n\nnamespace hm {\n\n')
    with open(OUT, "w") as f:
        f.write(hdr + "\n".join(funcs) + "\n}  // namespace hm\n")
    print(OUT)


if __name__ == "__main__":
    main()
