"""The reference's FlatFileIO ascii layout (src/FileIO/FlatFileIO.cc), read
for the tests: one "path value" line per written value; Fields are
"path n v0 v1 ...", vectors and tensors "( a b c )", FieldLists write
path/NodeListNames ("name|" and a NUL) then path/Field0."""
import numpy as np


def entries(data):
    """[(path, raw value bytes)] in file order."""
    out = []
    for line in data.split(b"\n"):
        if not line:
            continue
        path, _, rest = line.partition(b" ")
        out.append((path.decode(), rest))
    return out


def labels(data):
    """The object labels (first path component) in order of first appearance."""
    seen = []
    for path, _ in entries(data):
        lab = path.split("/")[0]
        if lab not in seen:
            seen.append(lab)
    return seen


def numbers(raw):
    """The numbers of a value ("(" and ")" skipped)."""
    toks = [t for t in raw.split() if t not in (b"(", b")")]
    return np.array([float(t) for t in toks], dtype=np.float64)


def field(raw):
    """A Field's values (the leading node count dropped), as a flat array."""
    v = numbers(raw)
    n, rest = int(v[0]), v[1:]
    assert (n == 0 and rest.size == 0) or (n > 0 and rest.size % n == 0)
    return rest


def as_dict(data):
    return dict(entries(data))
