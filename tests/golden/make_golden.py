"""Build tests/golden/*.npz from the evoc-rs golden fixtures.

Run once in a container where the reference tree is mounted:

    python tests/golden/make_golden.py [/path/to/evoc-rs]

The reference's fixtures (tests/fixtures/{small_200,medium_800,large_2000}) were
produced by upstream Python EVoC (scripts/generate_parity_fixtures.py:18-25,
156-160 in evoc-rs) and are the golden vectors its own parity suites use:
  tests/parity.rs:34-68,134-260     kNN indices/distances (assert_knn_parity rules)
  tests/graph_parity.rs:28-90       sigma/rho and the fuzzy-union graph
  tests/parity_intermediates.rs:655-687  NumPy RNG state after knn_graph
The arrays are copied unchanged into one compressed .npz per fixture so the
tests can run where the reference tree is absent.

lp_<fixture>.npz carries the label-propagation and node-embedding goldens
(tests/parity_intermediates.rs:46-135,327-375,405-457,593-653 read the same
intermediates): per-iteration labels, the partition, the reduced data/graph,
init and layout, the final init_embedding and embedding, NumPy RNG states
between the stages, and (large_2000) the reference's own Rust node orders and
embedding state after 20 reproducible epochs (rust_*_after19.npy); and
(medium_800) the KD-tree index order, core distances and Borůvka MST edges
Python computed on its final embedding.
"""
import json
import os
import sys

import numpy as np

# The evoc-rs checkout: the first argument, else $EVOC_REFERENCE_TREE, else /root/reference.
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EVOC_REFERENCE_TREE", "/root/reference")
OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    root = os.path.join(REF, "tests", "fixtures")
    summary = json.load(open(os.path.join(root, "summary.json")))
    for name in ("small_200", "medium_800", "large_2000"):
        d = os.path.join(root, name)
        inter = os.path.join(d, "intermediates")
        arrs = {
            "data": np.load(os.path.join(d, "data.npy")),
            "nn_inds": np.load(os.path.join(d, "nn_inds.npy")),
            "nn_dists": np.load(os.path.join(d, "nn_dists.npy")),
            "rng_after_knn_key": np.load(os.path.join(inter, "rng_after_knn_key.npy")),
            "seed": np.array(summary[name]["seed"], np.int64),
        }
        meta = np.load(os.path.join(inter, "rng_after_knn_meta.npz"))
        arrs["rng_after_knn_pos"] = meta["pos"]
        for g in ("graph_coo", "graph_csr"):
            p = os.path.join(inter, g + ".npz")
            if os.path.exists(p):
                z = np.load(p)
                for key in z.files:
                    arrs[f"{g}_{key}"] = z[key]
        for f in ("sigmas_py", "rhos_py", "sigmas", "rhos"):
            p = os.path.join(inter, f + ".npy")
            if os.path.exists(p):
                arrs[f] = np.load(p)
        p = os.path.join(d, "leaf_array.npy")
        if os.path.exists(p):
            arrs["leaf_array"] = np.load(p)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **arrs)
        print(name, {k: v.shape for k, v in arrs.items()})
        lp = label_prop_arrays(inter)
        np.savez_compressed(os.path.join(OUT, f"lp_{name}.npz"), **lp)
        print("lp_" + name, sorted(lp))


LP_ARRAYS = ["labels_seeded", "labels_iter0", "labels_iter1", "labels_iter2", "labels_iter5", "labels_iter10",
             "labels_iter19", "labels_after_outliers", "partition", "reduced_data", "reduced_init", "reduced_layout",
             "pre_scale_result", "init_embedding", "embedding", "rust_emb_after19", "rust_updates_after19",
             "rust_eon_after19", "rust_eos_after19", "rust_node_order_000", "rust_node_order_012",
             "rust_node_order_024", "py_kdtree_idx_array", "py_core_distances", "py_boruvka_edges"]
LP_CSR = ["graph_csr", "reduced_graph_csr", "temp_norm_t_graph"]
LP_RNG = ["after_knn", "after_partition", "after_reduced_init", "after_init", "after_emb"]


def label_prop_arrays(inter):
    out = {}
    for f in LP_ARRAYS:
        p = os.path.join(inter, f + ".npy")
        if os.path.exists(p):
            out[f] = np.load(p)
    for f in LP_CSR:
        p = os.path.join(inter, f + ".npz")
        if os.path.exists(p):
            z = np.load(p)
            for key in ("indptr", "indices", "data", "shape"):
                out[f"{f}_{key}"] = z[key]
    for tag in LP_RNG:
        p = os.path.join(inter, f"rng_{tag}_key.npy")
        if os.path.exists(p):
            meta = np.load(os.path.join(inter, f"rng_{tag}_meta.npz"))
            out[f"rng_{tag}_key"] = np.load(p)
            out[f"rng_{tag}_pos"] = meta["pos"]
            out[f"rng_{tag}_has_gauss"] = meta["has_gauss"]
            out[f"rng_{tag}_gauss"] = meta["gauss"]
    return out


if __name__ == "__main__":
    main()
