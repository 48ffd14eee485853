"""Extract the reference's median-filter known answer into ``median_golden.json``.

The reference test ``tests/test_denoiser.py`` (``test_median_filter_3d``) filters ``np.arange(27).reshape(3, 3,
3)`` and compares with a literal 3x3x3 array.  This script reads that file as text (it is never imported or
executed), pulls the literal out with ``ast``, and writes input and expected output as a fixture.

Usage: python tests/golden/make_median_golden.py <path/to/reference/root>  (or MBIRJAX_REFERENCE_ROOT=<root>)
"""
import ast
import json
import os
import sys


def extract(reference_root):
    path = os.path.join(reference_root, 'tests', 'test_denoiser.py')
    tree = ast.parse(open(path).read())
    func = next(n for n in ast.walk(tree) if isinstance(n, ast.FunctionDef) and n.name == 'test_median_filter_3d')
    expected = None
    for stmt in func.body:
        if (isinstance(stmt, ast.Assign) and len(stmt.targets) == 1 and isinstance(stmt.targets[0], ast.Name)
                and isinstance(stmt.value, ast.Call) and stmt.value.args):
            try:
                val = ast.literal_eval(stmt.value.args[0])
            except ValueError:
                continue
            if isinstance(val, list) and len(val) == 3:
                expected = val
    if expected is None:
        raise RuntimeError('no 3x3x3 literal found in %s' % path)
    return {'input': 'np.arange(27).reshape(3, 3, 3)', 'expected': expected,
            'source': 'reference tests/test_denoiser.py (test_median_filter_3d)'}


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MBIRJAX_REFERENCE_ROOT')
    if not root:
        sys.exit('usage: %s <mbirjax reference root> (or set MBIRJAX_REFERENCE_ROOT)' % sys.argv[0])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'median_golden.json')
    with open(out, 'w') as f:
        json.dump(extract(root), f, indent=1)
    print('wrote', out)
