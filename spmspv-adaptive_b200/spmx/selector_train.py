"""Train the kernel selector on this hardware and export it as C++.

Follows the reference's offline pipeline (model/1-generate_matrix_class.py:
label = the fastest kernel; model/1-test_dtree.py: a DecisionTreeClassifier
chosen by GridSearchCV over criterion and depth on a 70/30 split with
random_state=4; get_code, :93-112, prints the tree as if/else), with three
differences:
  - one tree over the eight kernels instead of three chained trees;
  - the inputs are exactly what spmx_select sees at run time without a device
    round trip (spmx_selector_inputs: matrix features, x_nnz, bin_len
    estimated as x_nnz*nnz/n, the matrix's longest column);
  - the labels come from timing all eight kernels on the GPU here
    (`collect`), the split and the fit run on the host (`fit`).

usage:
  python -m spmx.selector_train collect OUT.jsonl [A.mtx ...]   (GPU)
  python -m spmx.selector_train features OUT.jsonl A.mtx ...    (GPU)
  python -m spmx.selector_train fit DATA.jsonl OUT.inc          (host, scikit-learn)
  python -m spmx.selector_train compare DATA.jsonl              (host: other learners)

`collect` times all eight kernels on the synthetic spread below, or on the
given MatrixMarket files (the reference's generate_model_data.cu:563-860 does
the same over its matrix list).  `features` writes one JSON line of matrix
features per file (generate_feature.cu:209-290 writes the same fields as a
text line).
"""
import json
import math
import statistics
import sys

import numpy as np

from ._lib import FEATURE_NAMES, KERNEL_NAMES, NUM_KERNELS

DENSITIES = [1e-6, 3e-6, 1e-5, 3e-5, 1e-4, 3e-4, 1e-3, 3e-3, 1e-2, 2e-2, 5e-2, 0.1, 0.2, 0.35,
             0.5, 0.75, 1.0]


def matrices():
    """(name, Csr) pairs: the benchmark's shapes and a spread around them."""
    from . import gen
    yield "zipf-1M", gen.zipf_rows(1 << 20, 1.5, 16, 10000, seed=2)
    yield "zipf-256K", gen.zipf_rows(1 << 18, 1.5, 16, 10000, seed=12)
    yield "zipf-1M-mean4", gen.zipf_rows(1 << 20, 1.5, 4, 10000, seed=13)
    yield "zipf-512K-mean64", gen.zipf_rows(1 << 19, 1.5, 64, 10000, seed=14)
    for sc in (16, 20):
        g = gen.rmat(sc, 16, seed=sc)
        g.val = np.random.default_rng(sc).uniform(-1, 1, g.nnz).astype(np.float32)
        yield f"rmat-{sc}", g
    yield "chunglu-1M", gen.chung_lu(1 << 20, 2.1, 32.0, seed=5)
    yield "laplacian-1024", gen.laplacian(1024, 0.01, seed=4)
    yield "laplacian-2048", gen.laplacian(2048, 0.01, seed=4)


def mtx_matrices(paths):
    """(name, Csr) pairs read from MatrixMarket files: host parse, GPU sort."""
    import os
    from . import io
    from .gen import Csr
    for p in paths:
        h = io.load_mtx(p)
        rp, cl, vl = (t.cpu().numpy() for t in h.get_csr())
        h.Destroy()
        yield os.path.basename(p), Csr(h.m, h.n, rp, cl, vl)


MAT_FEATURES = ("m", "n", "nnz", "maxRow", "minRow", "avgRow", "range", "stdRow",
                "edge_equlity", "gini_coefficiency")


def dump_features(out_path, paths):
    """One JSON line of matrix features per MatrixMarket file."""
    import os
    from . import io
    with open(out_path, "w") as out:
        for p in paths:
            h = io.load_mtx(p)
            f = dict(zip(MAT_FEATURES, h.computeMatFeture()))
            h.Destroy()
            out.write(json.dumps({"matrix": os.path.basename(p), **f}) + "\n")
            out.flush()


def collect(out_path, reps=7, paths=None):
    import torch
    from .handle import SpmspvHandle
    from . import gen
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(64 << 20, device=dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with open(out_path, "w") as out:
        for name, A in (mtx_matrices(paths) if paths else matrices()):
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
            vals = A.val if A.val is not None else np.ones(A.nnz, np.float32)
            rp, cl, vl = t(A.rowptr), t(A.col), t(vals)
            h = SpmspvHandle(A.m, A.n, A.nnz, stream=stream)
            h.InputCSR(A.nnz, rp, cl, vl)
            h.ToCSC()
            h.allocPreBuffer()
            backend = h.autotune()
            y = torch.empty(A.m, device=dev)
            for d in DENSITIES:
                k = gen.density_nnz(A.n, d)
                if k == 0:
                    continue
                key, val = gen.sparse_vector(A.n, k, seed=77 + k)
                kd, vd = t(key), t(val)
                h.set_sparse_x(kd, vd, k)
                inputs = h.selector_inputs()
                exact = h.features()
                times = []
                for kid in range(NUM_KERNELS):
                    ts = []
                    for it in range(reps + 2):
                        flush.fill_(float(it))
                        s.record(stream)
                        h.run_kernel(kid, 1.0, y)
                        e.record(stream)
                        stream.synchronize()
                        if it >= 2:
                            ts.append(s.elapsed_time(e) * 1e3)
                    times.append(statistics.median(ts))
                h.check_device_error()
                rec = {"matrix": name, "density": d, "x_nnz": k, "spmv_backend": backend,
                       "inputs": inputs,
                       "features": [exact[n_] for n_ in FEATURE_NAMES], "us": times,
                       "best": int(np.argmin(times))}
                out.write(json.dumps(rec) + "\n")
                out.flush()
                print(name, d, KERNEL_NAMES[rec["best"]], [round(x, 1) for x in times], flush=True)
            h.Destroy()


# host-known inputs the tree may split on (indices into the 23-entry schema);
# "min" (13) is not known without a device pass and is left out
TREE_FEATURES = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 14, 15, 16, 17, 18, 19, 20, 21, 22]


def _load(path):
    recs = [json.loads(ln) for ln in open(path) if ln.strip()]
    X = np.array([[r["inputs"][i] for i in TREE_FEATURES] for r in recs], np.float64)
    T = np.array([r["us"] for r in recs], np.float64)
    return recs, X, T


class _RegressionPick:
    """A multi-output regression tree on log-times wrapped as a classifier:
    each leaf picks the kernel with the smallest mean log-time."""

    def __init__(self, reg):
        self.reg = reg
        self.tree_ = getattr(reg, "tree_", None)  # set again after fitting
        self.classes_ = np.arange(NUM_KERNELS)

    def predict(self, X):
        return np.argmin(self.reg.predict(X), axis=1)

    def leaf_label(self, node):
        return int(np.argmin(self.tree_.value[node][:, 0]))


def _cv_pick(make, grid, X, T, fit_kw, folds=5, seed=4):
    """The hyper-parameters with the lowest mean cross-validated regret."""
    from sklearn.model_selection import KFold
    best, best_r = None, None
    kf = KFold(n_splits=min(folds, len(X)), shuffle=True, random_state=seed)
    for params in grid:
        rs = []
        for a, b in kf.split(X):
            m = make(params)
            fit_kw(m, X[a], T[a])
            p = m.predict(X[b])
            rs.append(float(np.mean(T[b, p] / T[b].min(axis=1))))
        r = float(np.mean(rs))
        if best_r is None or r < best_r - 1e-12:
            best, best_r = params, r
    return best, best_r


def fit(data_path, out_inc, report=True):
    """Fit a classification tree (the reference's model) and a multi-output
    regression tree on log kernel times, each with the hyper-parameters of the
    lowest cross-validated regret on a 70/30 split (random_state=4, as the
    reference's model/1-test_dtree.py); keep the one with the lower held-out
    regret, then refit it on every case for export."""
    from sklearn.model_selection import train_test_split
    from sklearn.tree import DecisionTreeClassifier, DecisionTreeRegressor
    recs, X, T = _load(data_path)
    y = T.argmin(axis=1)
    idx = np.arange(len(y))
    tr, te = train_test_split(idx, test_size=0.3, random_state=4)

    def make_clf(p):
        return DecisionTreeClassifier(random_state=4, **p)

    def fit_clf(m, Xa, Ta):
        # sample weight: what a wrong pick can cost
        m.fit(Xa, Ta.argmin(axis=1), sample_weight=Ta.max(axis=1) / Ta.min(axis=1))

    def make_reg(p):
        return _RegressionPick(DecisionTreeRegressor(random_state=4, **p))

    def fit_reg(m, Xa, Ta):
        m.reg.fit(Xa, np.log(Ta))
        m.tree_ = m.reg.tree_

    clf_grid = [{"criterion": c, "max_depth": d} for c in ("gini", "entropy") for d in range(1, 11)]
    reg_grid = [{"max_depth": d, "min_samples_leaf": l} for d in range(2, 13) for l in (1, 2, 4)]
    cp, _ = _cv_pick(make_clf, clf_grid, X[tr], T[tr], fit_clf)
    rp, _ = _cv_pick(make_reg, reg_grid, X[tr], T[tr], fit_reg)
    clf = make_clf(cp)
    fit_clf(clf, X[tr], T[tr])
    reg = make_reg(rp)
    fit_reg(reg, X[tr], T[tr])
    cands = {"classifier": (clf, cp, make_clf, fit_clf), "regressor": (reg, rp, make_reg, fit_reg)}

    def regret(model, ix):
        p = model.predict(X[ix])
        return float(np.mean(T[ix, p] / T[ix].min(axis=1)))

    kind = min(cands, key=lambda k: (regret(cands[k][0], te), regret(cands[k][0], tr)))
    held, params, make, fitter = cands[kind]
    stats = {"model": kind, "train_regret": regret(held, tr), "test_regret": regret(held, te),
             "test_accuracy": float(np.mean(held.predict(X[te]) == y[te])),
             "params": params, "n": int(len(y))}
    # the exported selector: the chosen model and hyper-parameters refitted
    # on every case (the held-out figures above describe the 70 % fit)
    tree = make(params)
    fitter(tree, X, T)
    stats["all_regret"] = regret(tree, idx)
    with open(out_inc, "w") as f:
        f.write(export_cpp(tree, stats))
    if report:
        print(json.dumps(stats))
    return tree, stats


def compare(data_path, report=True):
    """Held-out regret of other learners on the same 70/30 split, beside the
    decision tree (the reference compares SVM / GBDT / random forest in
    model/*.py).  Features are log-scaled for the distance- and kernel-based
    learners.  Only the tree is exported: it compiles to branches."""
    from sklearn.ensemble import GradientBoostingClassifier, RandomForestClassifier
    from sklearn.model_selection import train_test_split
    from sklearn.neighbors import KNeighborsClassifier
    from sklearn.pipeline import make_pipeline
    from sklearn.preprocessing import FunctionTransformer, StandardScaler
    from sklearn.svm import SVC
    from sklearn.tree import DecisionTreeClassifier
    recs, X, T = _load(data_path)
    y = T.argmin(axis=1)
    tr, te = train_test_split(np.arange(len(y)), test_size=0.3, random_state=4)
    w = T[tr].max(axis=1) / T[tr].min(axis=1)
    logx = FunctionTransformer(lambda a: np.log1p(np.abs(a)) * np.sign(a))
    learners = {
        "decision tree": (DecisionTreeClassifier(random_state=4, max_depth=6), True),
        "random forest": (RandomForestClassifier(n_estimators=200, random_state=4), True),
        "gradient boosting": (GradientBoostingClassifier(random_state=4), True),
        "svm (rbf)": (make_pipeline(logx, StandardScaler(), SVC(C=10.0, gamma="scale")), False),
        "k nearest (5)": (make_pipeline(logx, StandardScaler(), KNeighborsClassifier(5)), False),
    }
    out = {}
    for name, (model, weighted) in learners.items():
        if weighted:
            model.fit(X[tr], y[tr], sample_weight=w)
        else:
            model.fit(X[tr], y[tr])
        p = model.predict(X[te])
        out[name] = {"test_regret": float(np.mean(T[te, p] / T[te].min(axis=1))),
                     "test_accuracy": float(np.mean(p == y[te]))}
    best = T[te].min(axis=1)
    out["always the overall best kernel"] = {
        "test_regret": float(np.mean(T[te, np.bincount(y[tr]).argmax()] / best)), "test_accuracy": None}
    if report:
        print(json.dumps(out, indent=1))
    return out


def export_cpp(tree, stats):
    """The fitted tree as nested if/else over the feature vector."""
    t = tree.tree_
    lines = [
        "// Generated by spmx/selector_train.py (fit) from kernel timings measured on",
        "// B200; do not edit by hand.  Regret (time of the pick / time of the best",
        f"// kernel): 70/30 split train {stats['train_regret']:.3f}, held-out",
        f"// {stats['test_regret']:.3f}; refitted on all cases {stats['all_regret']:.3f} ({stats['model']});",
        f"// held-out accuracy {stats['test_accuracy']:.3f}; {stats['n']} (matrix, density) cases;",
        f"// {json.dumps(stats['params'])}.",
        "#pragma once",
        "namespace spmx {",
        "SPMX_HD inline int select_by_tree(const double* f) {",
    ]

    def rec(node, depth):
        pad = "  " * depth
        if t.children_left[node] == -1:
            if isinstance(tree, _RegressionPick):
                lab = tree.leaf_label(node)
            else:
                # leaf values are indexed like tree.classes_ (the labels seen in training)
                lab = int(tree.classes_[int(np.argmax(t.value[node][0]))])
            lines.append(f"{pad}return {lab};")
            return
        fi = TREE_FEATURES[t.feature[node]]
        lines.append(f"{pad}if (f[{fi}] <= {repr(float(t.threshold[node]))}) {{  // {FEATURE_NAMES[fi]}")
        rec(t.children_left[node], depth + 1)
        lines.append(f"{pad}}} else {{")
        rec(t.children_right[node], depth + 1)
        lines.append(f"{pad}}}")

    rec(0, 1)
    lines += ["}", "}  // namespace spmx", ""]
    return "\n".join(lines)


def main(argv):
    if len(argv) >= 2 and argv[0] == "collect":
        collect(argv[1], paths=argv[2:] or None)
    elif len(argv) >= 3 and argv[0] == "features":
        dump_features(argv[1], argv[2:])
    elif len(argv) >= 3 and argv[0] == "fit":
        fit(argv[1], argv[2])
    elif len(argv) >= 2 and argv[0] == "compare":
        compare(argv[1])
    else:
        print(__doc__)
        return 2
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
