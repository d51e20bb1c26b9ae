"""CPU checks of bench.py's reference arm: it must time the reference's own
sgemm() with nothing of this repository's library loaded (its inputs come from
the oracle's host generator), and both arms must describe the workload with
the same config except for the kernel that runs."""
import ast
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _functions():
    tree = ast.parse(open(os.path.join(ROOT, "bench.py")).read())
    return {f.name: f for f in tree.body if isinstance(f, ast.FunctionDef)}


def test_reference_arm_loads_nothing_of_the_library():
    fns = _functions()
    for name in ("run_reference", "_host_inputs", "_reference_config_1024"):
        f = fns[name]
        for node in ast.walk(f):
            if isinstance(node, (ast.Import, ast.ImportFrom)):
                mods = [a.name for a in node.names] + [getattr(node, "module", None) or ""]
                assert not any("sgemm_b200" in m for m in mods), (name, mods)
            if isinstance(node, ast.Name):
                assert node.id != "sg", f"{name} uses the library binding"
    # and every helper it calls is library-free too
    called = {n.func.id for n in ast.walk(fns["run_reference"])
              if isinstance(n, ast.Call) and isinstance(n.func, ast.Name)}
    for helper in called & set(fns):
        for node in ast.walk(fns[helper]):
            if isinstance(node, ast.Name):
                assert node.id != "sg", f"{helper} (called by the reference arm) uses the library"


def test_both_arms_build_config_with_the_same_function():
    fns = _functions()
    for name in ("run", "run_reference"):
        calls = [n for n in ast.walk(fns[name]) if isinstance(n, ast.Call)
                 and isinstance(n.func, ast.Name) and n.func.id == "_config"]
        assert calls, f"{name} does not build its config with _config"


def test_both_arms_sweep_the_reference_square_sizes():
    """The sweep legs of both arms run the same sizes: 1024..16384 in steps of
    1024 plus the sizes that are not multiples of a tile (1000, 3001, 5003)."""
    src = open(os.path.join(ROOT, "bench.py")).read()
    tree = ast.parse(src)
    sizes = None
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "SWEEP_SIZES"
                                                for t in node.targets):
            sizes = eval(compile(ast.Expression(node.value), "bench.py", "eval"))
    assert sizes == sorted([1000, 3001, 5003] + list(range(1024, 16385, 1024)))
    fns = _functions()
    for name, leg in (("run", "_sweep_leg"), ("run_reference", "_reference_sweep")):
        calls = [n for n in ast.walk(fns[name]) if isinstance(n, ast.Call)
                 and isinstance(n.func, ast.Name) and n.func.id == leg]
        assert calls and any(isinstance(a, ast.Name) and a.id == "SWEEP_SIZES"
                             for c in calls for a in c.args), name
