"""Binary graph and update-stream files (readers in libdycg and the CLI).

Graph, "DYCGCSR1" (little-endian):
    char magic[8]; uint64 n; uint64 m; uint64 flags (bit 0: weights present)
    uint64 offsets[n+1]; uint32 dst[m]; uint32 w[m] (if bit 0)
Update stream, "DYCGUPD1":
    char magic[8]; uint64 snapshots; uint64 records; uint64 reserved
    uint32 sizes[snapshots][2]   (adds, dels) per snapshot, the reference's sizes file
    dycg_edge records[records]   per snapshot: its dels, then its adds (12 bytes each)
These replace the text formats (src/utils/parser.cpp:296-406 market_big,
include/framework/Loader.h:30-101 update lines) for graphs that do not parse in
seconds as text.
"""
import numpy as np

GRAPH_MAGIC = b"DYCGCSR1"
UPD_MAGIC = b"DYCGUPD1"


def write_graph(path, offsets, dst, w=None):
    offsets = np.ascontiguousarray(offsets, np.uint64)
    dst = np.ascontiguousarray(dst, np.uint32)
    n = offsets.shape[0] - 1
    with open(path, "wb") as f:
        f.write(GRAPH_MAGIC)
        np.array([n, dst.shape[0], 1 if w is not None else 0], np.uint64).tofile(f)
        offsets.tofile(f)
        dst.tofile(f)
        if w is not None:
            np.ascontiguousarray(w, np.uint32).tofile(f)


def read_graph(path):
    raw = np.memmap(path, dtype=np.uint8, mode="r")
    if bytes(raw[:8]) != GRAPH_MAGIC:
        raise ValueError("not a DYCGCSR1 file")
    n, m, flags = np.frombuffer(raw[8:32], np.uint64)
    o = 32
    off = np.frombuffer(raw[o:o + (n + 1) * 8], np.uint64)
    o += (n + 1) * 8
    dst = np.frombuffer(raw[o:o + m * 4], np.uint32)
    w = np.frombuffer(raw[o + m * 4:o + 2 * m * 4], np.uint32) if flags & 1 else None
    return int(n), off, dst, w


def write_updates(path, batches):
    """batches: list of (dels, adds) arrays of (u, v, w) rows."""
    sizes = np.array([[len(a), len(d)] for d, a in batches], np.uint32).reshape(-1, 2)
    recs = [np.asarray(x, np.uint32).reshape(-1, 3) for d, a in batches for x in (d, a)]
    allr = np.concatenate(recs) if recs else np.zeros((0, 3), np.uint32)
    with open(path, "wb") as f:
        f.write(UPD_MAGIC)
        np.array([len(batches), allr.shape[0], 0], np.uint64).tofile(f)
        sizes.tofile(f)
        allr.tofile(f)


def read_updates(path):
    raw = np.fromfile(path, np.uint8)
    if bytes(raw[:8]) != UPD_MAGIC:
        raise ValueError("not a DYCGUPD1 file")
    nb, nr, _ = np.frombuffer(raw[8:32], np.uint64)
    sizes = np.frombuffer(raw[32:32 + nb * 8], np.uint32).reshape(-1, 2)
    recs = np.frombuffer(raw[32 + nb * 8:32 + nb * 8 + nr * 12], np.uint32).reshape(-1, 3)
    out, p = [], 0
    for na, nd in sizes:
        out.append((recs[p:p + nd], recs[p + nd:p + nd + na]))
        p += nd + na
    return out


def read_text_updates(update_path, sizes_path):
    """Text update stream -> [(dels, adds), ...] per snapshot, split as the
    reference's Loader splits it (include/framework/Loader.h:30-101): each
    sizes line "adds dels" takes the next adds 'a' records and the next dels
    'd' records in file order; an update line is "t u v [w]" (t in {a, d}; w
    defaults to 1, other lines are skipped)."""
    sizes = []
    with open(sizes_path) as f:
        for line in f:
            p = line.split()
            if len(p) >= 2 and p[0].isdigit() and p[1].isdigit():
                sizes.append((int(p[0]), int(p[1])))
    recs = {"a": [], "d": []}
    with open(update_path) as f:
        for line in f:
            p = line.split()
            if len(p) < 3 or p[0] not in recs or not (p[1].isdigit() and p[2].isdigit()):
                continue
            w = int(p[3]) if len(p) > 3 and p[3].isdigit() else 1
            recs[p[0]].append((int(p[1]), int(p[2]), w))
    batches, ia, idl = [], 0, 0
    for na, nd in sizes:
        batches.append((np.asarray(recs["d"][idl:idl + nd], np.uint32).reshape(-1, 3),
                        np.asarray(recs["a"][ia:ia + na], np.uint32).reshape(-1, 3)))
        ia += na
        idl += nd
    return batches


def text_updates_to_binary(update_path, sizes_path, out_path):
    """Text update stream + sizes file -> DYCGUPD1 (read_text_updates' split).
    Returns the number of snapshots written."""
    batches = read_text_updates(update_path, sizes_path)
    write_updates(out_path, batches)
    return len(batches)


def main(argv=None):
    """python -m dycgraph_b200.formats graph TEXT OUT [--weighted] [--min-nodes N]
    converts a text edge list (the reference's market_big lines) to the binary
    graph file, parsed by the library exactly as its text loader does;
    python -m dycgraph_b200.formats updates UPDATES SIZES OUT converts a text
    update stream and its sizes file to the binary update stream."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m dycgraph_b200.formats")
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("graph", help="text edge list -> DYCGCSR1")
    g.add_argument("text")
    g.add_argument("out")
    g.add_argument("--weighted", action="store_true", help="read a third column as weights")
    g.add_argument("--min-nodes", type=int, default=0)
    u = sub.add_parser("updates", help="text update stream + sizes file -> DYCGUPD1")
    u.add_argument("updates")
    u.add_argument("sizes")
    u.add_argument("out")
    args = ap.parse_args(argv)
    if args.cmd == "updates":
        nb = text_updates_to_binary(args.updates, args.sizes, args.out)
        print(f"{args.out}: {nb} snapshots")
        return
    from .engine import convert_graph_text
    convert_graph_text(args.text, args.out, args.min_nodes, args.weighted)
    n, off, dst, w = read_graph(args.out)
    print(f"{args.out}: {n} vertices, {len(dst)} edges{', weighted' if w is not None else ''}")


if __name__ == "__main__":
    main()
