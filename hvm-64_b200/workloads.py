"""Seeded synthetic workloads for net normalisation, emitted as `.hvm` text.

Families (each a Book whose `@main` is the net to normalise):

  tree_sum(depth, seed)   `gen(depth, 0)` builds a complete Scott-encoded
                          binary tree whose leaf i holds mix24(i); `sum` folds
                          it with OPER add (u24, wrapping).  Normal form: one
                          u24 number, checked against `expected_sum`.
  bitonic(depth, seed)    the same generator with keys mix24(i) mod (10*2^d)
                          (about 5% duplicate keys), sorted by the bitonic
                          sorter; normal form: the sorted leaf tree.
  church(k, last)         Church numeral 2 with a distinct DUP label per copy,
                          applied to itself k times and collapsed by applying
                          the result to CON-encoded lambda f. lambda x. x.

The sum / sort / Leaf / Node definitions are the reference's own example
programs (tests/programs/stress_tests/sum_tree.hvm and
examples/sort/bitonic/bitonic_sort_lam.hvm, read from the golden fixtures);
only `@gen`'s leaf and `@main` change.  Leaf values come from an in-net u24
mixer because u24 arithmetic cannot carry xorshift64:

  mix24(i) = f2(K2 * f1(K1 * (i ^ s)))  with  f1(t) = t ^ (t >> 12),
             f2(u) = u ^ (u >> 11), all mod 2^24, s = splitmix64(BASE + j) & 0xFFFFFF.

Seeds: BASE = 0x9E3779B97F4A7C15; net j uses splitmix64(BASE + j).
"""
import json
import math
import os
import random

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(ROOT, "tests", "golden", "programs.json")

BASE_SEED = 0x9E3779B97F4A7C15
K1 = 0x9E3779
K2 = 0x5BD1E9
M24 = (1 << 24) - 1


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & (2**64 - 1)
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
    return z ^ (z >> 31)


def seed24(j):
    return splitmix64(BASE_SEED + j) & M24


def mix24(i, s):
    t = ((i ^ s) * K1) & M24
    t ^= t >> 12
    u = (t * K2) & M24
    return u ^ (u >> 11)


_templates = None


def _template(name):
    global _templates
    if _templates is None:
        _templates = {p["name"]: p["source"] for p in json.load(open(GOLDEN))}
    return _templates[name]


def _defs(src, drop):
    """Split a book into {name: body text} and drop the listed defs."""
    out, cur, body = {}, None, []
    for line in src.splitlines():
        if line.startswith("@") and "=" in line:
            if cur is not None:
                out[cur] = "\n".join(body)
            cur = line.split("=", 1)[0].strip()[1:]
            body = [line]
        elif cur is not None:
            body.append(line)
    if cur is not None:
        out[cur] = "\n".join(body)
    return {k: v for k, v in out.items() if k not in drop}


GEN = """@gen = (?((a b) c) c)
& (a b) ~ (@gen$S0 @gen$S1)
@gen$S0 = (a b)
& @Leaf ~ (c b)
& @mix ~ (a c)
@gen$S1 = (#3{a b} (#4{$([*2] c) $([*2] $([+1] d))} e))
& @Node ~ (f (g e))
& @gen ~ (b (d g))
& @gen ~ (a (c f))"""


def tree_sum(depth, seed=0):
    """Book text for the tree-sum workload of `depth` (root `@main`)."""
    s = seed24(seed)
    base = _defs(_template("examples::sort::bitonic::bitonic_sort_lam"),
                 drop={"main", "gen", "gen$S0", "gen$S1", "sort", "sort$S0", "sort$S1"})
    keep = {k: v for k, v in base.items() if k in ("Leaf", "Node", "sum", "sum$S0")}
    mix = (f"@mix = ($([^{s}] $([*{K1}] #9{{$([^] $(d $([*{K2}] #9{{$([^] $(g y)) $([:>>11] g)}})))"
           f" $([:>>12] d)}})) y)")
    main = f"@main = a\n& @sum ~ (b a)\n& @gen ~ ({depth} (0 b))"
    return "\n".join(list(keep.values()) + [GEN, mix, main]) + "\n"


def expected_sum(depth, seed=0):
    s = seed24(seed)
    return sum(mix24(i, s) for i in range(1 << depth)) & M24


def sort_keys(depth, seed=0):
    s = seed24(seed)
    mod = 10 << depth
    return [mix24(i, s) % mod for i in range(1 << depth)]


def bitonic(depth, seed=0, with_sum=False):
    """Book text for the bitonic-sort workload of `depth` (2^depth keys)."""
    s = seed24(seed)
    mod = 10 << depth
    src = _template("examples::sort::bitonic::bitonic_sort_lam")
    keep = _defs(src, drop={"main", "gen", "gen$S0", "gen$S1", "rev", "rev$S0", "rev$S1"})
    mix = (f"@mix = ($([^{s}] $([*{K1}] #9{{$([^] $(d $([*{K2}] #9{{$([^] $(g $([:%{mod}] y))) "
           f"$([:>>11] g)}}))) $([:>>12] d)}})) y)")
    if with_sum:
        main = f"@main = a\n& @sum ~ (b a)\n& @sort ~ (c (0 b))\n& @gen ~ ({depth} (0 c))"
    else:
        main = f"@main = a\n& @sort ~ (c (0 a))\n& @gen ~ ({depth} (0 c))"
    return "\n".join(list(keep.values()) + [GEN, mix, main]) + "\n"


def expected_bitonic_sum(depth, seed=0):
    return sum(sort_keys(depth, seed)) & M24


def church(k=5, last=2):
    """Church numerals with one DUP label per copy, applied to one another
    (tests/programs/stress_tests/boom.hvm shape) and collapsed by applying the
    result to lambda f. lambda x. x.  `k` copies of the numeral 2, except the
    last, which is the numeral `last`: value last ** (2 ** 2 ** ... ) built
    lazily; the collapse keeps only the tower below the top."""
    def numeral(n, lab):
        # n = lambda f. lambda x. f^n x, with f duplicated n-1 times (label lab)
        if n == 1:
            return f"((a R) (a R))"
        vs = [f"v{i}" for i in range(n + 1)]
        fs = f"(v1 v0)"
        for i in range(1, n):
            fs = f"#{lab}{{{fs} (v{i + 1} v{i})}}"
        return f"({fs} (v{n} v0))"
    defs = []
    for i in range(1, k + 1):
        defs.append(f"@n{i} = " + numeral(2 if i < k else last, i))
    defs.append("@F = (* (x x))")
    arg = "(@F R)"
    for i in range(k, 1, -1):
        arg = f"(@n{i} {arg})"
    defs.append(f"@main = R\n& @n1 ~ {arg}")
    return "\n".join(defs) + "\n"


CHURCH_BIG_NORMAL_FORM = "(* (a a))"


def church_big(nums=(2, 2, 2, 3)):
    """The label-heavy Church net at 10^8-10^9 interactions.  Numerals with
    one DUP label each (#1 .. #k) are applied to one another as in `church`:
    n1 n2 n3 n4 = n4^(n3^(n2^n1)) = 3^16 for (2, 2, 2, 3).  Instead of the
    eraser collapse (which discards almost all of the tower), the result is
    forced the way tests/programs/stress_tests/boom.hvm forces its tower:
    applied to `not` (@N = ((@F (@T a)) a)) and `true` (@T), so every one of
    the 3^16 applications runs.  3^16 is odd: the normal form is `false`,
    (* (a a)).  344,373,957 interactions (oracle)."""
    def numeral(n, lab):
        if n == 1:
            return "((a R) (a R))"
        fs = "(v1 v0)"
        for i in range(1, n):
            fs = f"#{lab}{{{fs} (v{i + 1} v{i})}}"
        return f"({fs} (v{n} v0))"
    defs = [f"@n{i + 1} = " + numeral(v, i + 1) for i, v in enumerate(nums)]
    defs += ["@F = (* (x x))", "@T = (a (* a))", "@N = ((@F (@T a)) a)"]
    arg = "(@N (@T R))"
    for i in range(len(nums), 1, -1):
        arg = f"(@n{i} {arg})"
    defs.append(f"@main = R\n& @n1 ~ {arg}")
    return "\n".join(defs) + "\n"


def leaves(text):
    """Leaf values of a read-back Scott tree, left to right (Leaf x prints as
    `((x a) (* a))`, Node l r as `(* ((l' (r' b)) b))`)."""
    import re
    return [int(m) for m in re.findall(r"\(\((\d+) [a-z]+\) \(\* [a-z]+\)\)", text)]


def batch_entries(n=4096, dmin=8, dmax=18, seed=0):
    """The uneven batch: net j is a tree-sum or a bitonic sort (50/50 by
    seed) of depth drawn log-uniform in [dmin, dmax]."""
    rng = random.Random(splitmix64(BASE_SEED ^ seed))
    out = []
    for j in range(n):
        kind = "sum" if (splitmix64(BASE_SEED + j) >> 7) & 1 else "sort"
        d = int(round(math.exp(rng.uniform(math.log(dmin), math.log(dmax)))))
        out.append((kind, max(dmin, min(dmax, d)), j))
    return out


def _family_defs():
    """Shared defs of both families (Leaf, Node, sum, sort and its helpers)."""
    src = _template("examples::sort::bitonic::bitonic_sort_lam")
    return _defs(src, drop={"main", "gen", "gen$S0", "gen$S1", "rev", "rev$S0", "rev$S1"})


def _net_defs(kind, depth, j):
    """Per-net generator defs (`@gen_j`, `@mix_j`) and the entry `@main_j`."""
    s = seed24(j)
    tail = f"$([:%{10 << depth}] y)" if kind == "sort" else "y"
    g = GEN.replace("@gen$S0", f"@gen_{j}$S0").replace("@gen$S1", f"@gen_{j}$S1").replace("@gen ", f"@gen_{j} ")
    g = g.replace("@mix ", f"@mix_{j} ")
    mix = (f"@mix_{j} = ($([^{s}] $([*{K1}] #9{{$([^] $(d $([*{K2}] #9{{$([^] $(g {tail})) $([:>>11] g)}})))"
           f" $([:>>12] d)}})) y)")
    if kind == "sum":
        main = f"@main_{j} = a\n& @sum ~ (b a)\n& @gen_{j} ~ ({depth} (0 b))"
    else:
        main = f"@main_{j} = a\n& @sort ~ (c (0 a))\n& @gen_{j} ~ ({depth} (0 c))"
    return "\n".join([g, mix, main])


def batch_book(entries):
    """One Book holding every net of a batch: shared family defs plus per-net
    generators; net j's entry point is `main_j`."""
    parts = list(_family_defs().values())
    for kind, depth, j in entries:
        parts.append(_net_defs(kind, depth, j))
    return "\n".join(parts) + "\n"


def check_result(kind, depth, j, text):
    """True when a net's read-back normal form is the expected answer."""
    if kind == "sum":
        return text == str(expected_sum(depth, j))
    return leaves(text) == sorted(sort_keys(depth, j))


def est_interactions(kind, depth):
    """Interaction count estimate per net (fitted on oracle runs)."""
    if kind == "sum":
        return 54 * (1 << depth)
    return (1 << depth) * depth * depth * (19.8 + 26.0 / depth)


def serving_requests(n, seed=0, lo=1e3, hi=1e8):
    """The serving stream's requests: (kind, param, j) with a target size drawn
    log-uniform in [lo, hi] interactions; kind tree-sum / bitonic sort /
    Church (47/47/6).  param is the depth (sum: up to 21, 1.1e8 interactions;
    sort: up to 14, 7e7) or (k, last) (Church: k = 4 below 1e5 interactions,
    else the 524,508-interaction k = 5)."""
    rng = random.Random(splitmix64(BASE_SEED ^ (0x5E4E + seed)))
    out = []
    for j in range(n):
        size = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        r = rng.random()
        if r < 0.47:
            d = max(3, min(21, int(round(math.log2(size / 54)))))
            out.append(("sum", d, j))
        elif r < 0.94:
            d = 2
            while d < 14 and est_interactions("sort", d) < size:
                d += 1
            out.append(("sort", d, j))
        else:
            out.append(("church", (4, 2 + j % 4) if size < 1e5 else (5, 2), j))
    return out


def est_request_interactions(kind, param):
    if kind == "church":
        return 6e4 if param[0] == 4 else 5.3e5
    return est_interactions(kind, param)


def est_request_nodes(kind, param):
    """A generous bound on a request's live heap nodes, for admission by node
    budget: an eighth of its interactions plus a floor."""
    return int(est_request_interactions(kind, param) / 8) + 4096


def serving_book(reqs):
    """One Book for a serving stream: the families' shared defs, per-request
    generators, and request j's entry point `main_j`."""
    parts = list(_family_defs().values())
    for kind, param, j in reqs:
        if kind == "church":
            k, last = param
            src = church(k, last)
            for i in range(k, 0, -1):
                src = src.replace(f"@n{i} ", f"@c{j}_n{i} ").replace(f"@n{i}\n", f"@c{j}_n{i}\n")
            src = src.replace("@F ", f"@c{j}_F ").replace("(@F ", f"(@c{j}_F ").replace("@main ", f"@main_{j} ")
            parts.append(src.strip())
        else:
            parts.append(_net_defs(kind, param, j))
    return "\n".join(parts) + "\n"


def check_request(kind, param, j, text):
    """True when a served request's normal form is its expected answer."""
    if kind == "church":
        return text == "(* (a a))"
    return check_result(kind, param, j, text)
