"""Generate tests/golden/reference_vectors.json from the reference crate's sources.

Run in a container that has the reference checkout (read-only) at REFERENCE_ROOT:

    python tests/golden/make_golden.py REFERENCE_ROOT   (or REFERENCE_ROOT=... in the env)

The reference is Rust and cannot be compiled here, so its golden data is read from
its source text:

* src/galois.rs:119-151      the 256-entry Backblaze log table and known products
* src/reedsolomon16.rs:1087-1101  the frozen GF((2^8)^2) wire vector (RS16(3,2))
* src/galois16.rs:194-196    the two structured const_matrix values
* src/gf/gfni.rs:83-87       affine matrices for c = 1 and c = 0
* src/fft_programs.rs        the generated LCH encode programs for six shapes: for
  each one, the header counts, a SHA-256 digest of the normalised op list, and the
  parity it produces on seeded random columns, evaluated here by replaying the
  reference's op list with an independent GF(2^8) multiply written in this file.

Only derived vectors and digests are written; no reference source is copied.
"""
import hashlib
import json
import os
import random
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def gf8_tables():
    """Independent GF(2^8) (poly 0x11d) tables, for replaying reference op lists."""
    exp = [0] * 512
    log = [0] * 256
    x = 1
    for i in range(255):
        exp[i] = x
        log[x] = i
        x <<= 1
        if x & 0x100:
            x ^= 0x11D
    for i in range(255, 512):
        exp[i] = exp[i - 255]
    return log, exp


LOG, EXP = gf8_tables()


def gmul(a, b):
    if a == 0 or b == 0:
        return 0
    return EXP[LOG[a] + LOG[b]]


def read(root, rel):
    with open(os.path.join(root, rel)) as f:
        return f.read()


def backblaze_table(src):
    m = re.search(r"BACKBLAZE_LOG_TABLE: \[u8; 256\] = \[(.*?)\];", src, re.S)
    return [int(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()]


def known_products(src):
    muls = [
        [int(a), int(b), int(c)]
        for a, b, c in re.findall(r"assert_eq!\(mul\((\d+), (\d+)\), (\d+)\);", src)
    ]
    exps = [
        [int(a), int(b), int(c)]
        for a, b, c in re.findall(r"assert_eq!\(exp\((\d+), (\d+)\), (\d+)\);", src)
    ]
    return muls, exps


def gf16_golden(src):
    body = src[src.index("fn golden_wire_vector"):]
    body = body[: body.index("\n    }\n")]
    shards = [
        [int(v, 16) for v in re.findall(r"0x([0-9a-fA-F]+)", row)]
        for row in re.findall(r"vec!\[(0x[^\]]*)\]", body)
    ]
    parity = [
        [int(v) for v in row.split(",")]
        for row in re.findall(r"assert_eq!\(shards\[\d\], \[([\d, ]+)\]", body)
    ]
    return {"k": 3, "m": 2, "data": shards, "parity": parity}


def fft_programs(src):
    shapes = [
        (int(a), int(b))
        for a, b in re.findall(
            r"\((\d+), (\d+)\),",
            src[src.index("GENERATED_SHAPES"): src.index("];", src.index("GENERATED_SHAPES"))],
        )
    ]
    out = []
    rng = random.Random(0x7A9E)
    for k, m in shapes:
        hdr = re.search(
            r"// shape \(%d,%d\): (\d+) registers, (\d+) ops, (\d+) multiplies" % (k, m), src
        )
        regs, n_ops, mults = (int(hdr.group(i)) for i in (1, 2, 3))
        start = src.index("macro_rules! fft_program_%d_%d" % (k, m))
        body = src[start: src.index("        );", start)]
        body = body[body.index("$off;") + len("$off;"):]
        ops = [" ".join(t.split()) for t in body.split(";") if t.strip()]
        digest = hashlib.sha256("\n".join(ops).encode()).hexdigest()
        # Replay the reference op list over seeded random columns.
        columns, parities = [], []
        for _ in range(64):
            col = [rng.randrange(256) for _ in range(k)]
            r = [0] * max(regs, k)
            par = [0] * m
            for op in ops:
                t = op.split()
                kind, a = t[0], [int(v) for v in t[1:]]
                if kind == "ld":
                    r[a[0]] = col[a[1]]
                elif kind == "mx":
                    r[a[0]] ^= gmul(a[2], r[a[1]])
                elif kind == "xo":
                    r[a[0]] ^= r[a[1]]
                elif kind == "mc":
                    r[a[0]] = gmul(a[2], r[a[1]])
                elif kind == "cp":
                    r[a[0]] = r[a[1]]
                elif kind == "st":
                    par[a[0]] = r[a[1]]
                else:
                    raise ValueError(op)
            columns.append(col)
            parities.append(par)
        n_body = sum(1 for o in ops if o.split()[0] not in ("ld", "st"))
        out.append(
            {
                "k": k,
                "m": m,
                "registers": regs,
                "ops_header": n_ops,
                "ops_body": n_body,
                "multiplies": mults,
                "sha256": digest,
                "columns": columns,
                "parity": parities,
            }
        )
    return out


def gfni_golden(src):
    vals = {}
    for c, v in re.findall(r"gfni_matrix\((\d+)\) as u64, (0x[0-9a-fA-F_]+u64|0)\)", src):
        vals[int(c)] = int(v.replace("_", "").replace("u64", ""), 0)
    return vals


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set REFERENCE_ROOT): the reference checkout")
    galois = read(root, "src/galois.rs")
    muls, exps = known_products(galois)
    g16 = read(root, "src/galois16.rs")
    cm = re.findall(r"assert_eq!\(const_matrix\((0x[0-9a-fA-F]+|\d+)\), \[([^\]]*)\]", g16)
    const_matrix = [
        [int(c, 0), [int(v) if v.strip().isdigit() else {"TOWER_L": 32}[v.strip()] for v in row.split(",")]]
        for c, row in cm
    ]
    errors = read(root, "src/errors.rs")
    variants = re.findall(r"^\s+(\w+),$", errors[errors.index("pub enum Error"): errors.index("}")], re.M)
    messages = dict(re.findall(r'Error::(\w+) => "([^"]*)"', errors))
    vectors = {
        "source": "spool-labs/reed-solomon (tape-reed-solomon 0.2.2), read as text",
        "error_variants": variants,
        "error_messages": [messages[v] for v in variants],
        "backblaze_log_table": backblaze_table(galois),
        "known_mul": muls,
        "known_exp": exps,
        "gf16_const_matrix": const_matrix,
        "gf16_tower_l": 32,
        "gf16_wire_vector": gf16_golden(read(root, "src/reedsolomon16.rs")),
        "gfni_matrix": gfni_golden(read(root, "src/gf/gfni.rs")),
        "fft_programs": fft_programs(read(root, "src/fft_programs.rs")),
    }
    path = os.path.join(HERE, "reference_vectors.json")
    with open(path, "w") as f:
        json.dump(vectors, f, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
