"""Insert-only cases shared by the golden-fixture generator and its CPU test."""
from csm import gen
from helpers import clique, star

CASES = (
    [dict(id=f"c1_seed{s}", config="c1", scale=1.0, seed=s, query=0, batch=1024, algorithms=[1, 2]) for s in
     (1001, 1002, 1003, 1004)]
    + [dict(id="c1_one_batch", config="c1", scale=1.0, seed=1001, query=0, batch=5000, algorithms=[1])]
    + [dict(id=f"c2small_q{q}", config="c2", scale=0.002, seed=1002, query=q, batch=500, algorithms=[1])
       for q in range(6)]
    + [dict(id="c1_triangle", config="c1", scale=1.0, seed=1001, query="triangle", batch=1024, algorithms=[1]),
       dict(id="c1_star3", config="c1", scale=0.2, seed=1001, query="star3", batch=250, algorithms=[1])]
)


def build_case(case):
    cfg = gen.scaled(case["config"], case["scale"]) if case["scale"] != 1.0 else dict(gen.CONFIGS[case["config"]])
    cfg["n_del"] = 0
    cfg["batch"] = case["batch"]
    w = gen.make_workload(case["config"], cfg, seed=case["seed"])
    q = case["query"]
    if q == "triangle":
        query = clique(3, label=0)
    elif q == "star3":
        query = star(3, center=1, leaf=0)
    else:
        query = w.queries[q]
    return query, w.data, w.batches, case["batch"]
