"""Writers of PCD test files (ascii, binary, binary_compressed with an LZF
stream of literal runs and back-references) for tests/test_pcd.py."""
import numpy as np


def lzf_compress(data: bytes) -> bytes:
    """Greedy LZF: literal runs of up to 32 bytes, back-references of 3-264
    bytes within 8 KB found through a table of 3-byte prefixes."""
    out, lit, table = bytearray(), bytearray(), {}
    i, n = 0, len(data)

    def flush():
        nonlocal lit
        while lit:
            chunk = lit[:32]
            out.append(len(chunk) - 1)
            out.extend(chunk)
            lit = lit[32:]

    while i < n:
        if i + 2 < n:
            key = bytes(data[i:i + 3])
            j = table.get(key)
            table[key] = i
            if j is not None and 0 < i - j <= 8192:
                L, maxl = 3, min(n - i, 264)
                while L < maxl and data[j + L] == data[i + L]:
                    L += 1
                flush()
                dist, ln = i - j - 1, L - 2
                if ln < 7:
                    out.append((ln << 5) | (dist >> 8))
                else:
                    out.append((7 << 5) | (dist >> 8))
                    out.append(ln - 7)
                out.append(dist & 0xFF)
                i += L
                continue
        lit.append(data[i])
        i += 1
    flush()
    return bytes(out)


def write_pcd(path, xyz: np.ndarray, mode: str, extra: bool = True):
    """Fields 'intensity x y z normal' (normal: COUNT 3) when extra, else
    'x y z'."""
    n = xyz.shape[0]
    rng = np.random.default_rng(n)
    inten = rng.uniform(0, 1, n).astype(np.float32)
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    if extra:
        fields, sizes, types, counts = ["intensity", "x", "y", "z", "normal"], [4] * 5, \
            ["F"] * 5, [1, 1, 1, 1, 3]
        cols = [inten[:, None], xyz[:, 0:1], xyz[:, 1:2], xyz[:, 2:3], nrm]
    else:
        fields, sizes, types, counts = ["x", "y", "z"], [4] * 3, ["F"] * 3, [1, 1, 1]
        cols = [xyz[:, 0:1], xyz[:, 1:2], xyz[:, 2:3]]
    head = ("# .PCD v.7 - Point Cloud Data file format\nVERSION .7\n"
            f"FIELDS {' '.join(fields)}\nSIZE {' '.join(map(str, sizes))}\n"
            f"TYPE {' '.join(types)}\nCOUNT {' '.join(map(str, counts))}\n"
            f"WIDTH {n}\nHEIGHT 1\nVIEWPOINT 0 0 0 1 0 0 0\nPOINTS {n}\nDATA {mode}\n")
    with open(path, "wb") as f:
        f.write(head.encode())
        if mode == "ascii":
            rec = np.concatenate(cols, 1)
            for r in rec:
                f.write((" ".join(repr(float(v)) for v in r) + "\n").encode())
        elif mode == "binary":
            rec = np.ascontiguousarray(np.concatenate(cols, 1).astype(np.float32))
            f.write(rec.tobytes())
        else:
            raw = b"".join(np.ascontiguousarray(c.astype(np.float32)).tobytes() for c in cols)
            comp = lzf_compress(raw)
            f.write(np.uint32(len(comp)).tobytes())
            f.write(np.uint32(len(raw)).tobytes())
            f.write(comp)
