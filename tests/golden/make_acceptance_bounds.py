"""Extract the reference's acceptance bounds into ``acceptance_bounds.json``.

The reference's end-to-end tests compare a reconstruction with its phantom and require the errors to stay under
literal bounds:

* ``tests/test_fbp_fdk.py``: ``self.fbp_tolerances`` and ``self.fdk_tolerances`` (max_diff, nrmse, pct_95);
* ``tests/test_vcd.py``: ``parallel_tolerances``, ``cone_tolerances`` and ``translation_tolerances``;
* ``tests/test_denoiser.py`` (``test_qggmrf_denoiser``) and ``tests/test_prox.py`` (``test_prox``): ``tolerance``.

This script reads those files as text (they are never imported or executed), pulls the literals out with
``ast``, and writes them as a fixture, so the tests here hold exactly the reference's numbers.

Usage: python tests/golden/make_acceptance_bounds.py <path/to/reference/root>  (or MBIRJAX_REFERENCE_ROOT=<root>)
"""
import ast
import json
import os
import sys


def _assigned_literals(path):
    """{name: literal} of every assignment of a literal in the file, to a name or to self.<name>."""
    out = {}
    for node in ast.walk(ast.parse(open(path).read())):
        if not (isinstance(node, ast.Assign) and len(node.targets) == 1):
            continue
        target = node.targets[0]
        if isinstance(target, ast.Attribute):
            name = target.attr
        elif isinstance(target, ast.Name):
            name = target.id
        else:
            continue
        try:
            out.setdefault(name, ast.literal_eval(node.value))
        except ValueError:
            continue
    return out


def _function_literal(path, func_name, name):
    tree = ast.parse(open(path).read())
    func = next(n for n in ast.walk(tree) if isinstance(n, ast.FunctionDef) and n.name == func_name)
    for node in ast.walk(func):
        if (isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name)
                and node.targets[0].id == name):
            return ast.literal_eval(node.value)
    raise RuntimeError('no literal %s in %s of %s' % (name, func_name, path))


def extract(reference_root):
    tests = os.path.join(reference_root, 'tests')
    fbp = _assigned_literals(os.path.join(tests, 'test_fbp_fdk.py'))
    vcd = _assigned_literals(os.path.join(tests, 'test_vcd.py'))
    return {
        'fbp': fbp['fbp_tolerances'],
        'fdk': fbp['fdk_tolerances'],
        'vcd': {'parallel': vcd['parallel_tolerances'], 'cone': vcd['cone_tolerances'],
                'translation': vcd['translation_tolerances']},
        'denoiser_nrmse': _function_literal(os.path.join(tests, 'test_denoiser.py'), 'test_qggmrf_denoiser',
                                            'tolerance'),
        'prox_max_diff': _function_literal(os.path.join(tests, 'test_prox.py'), 'test_prox', 'tolerance'),
        'source': 'reference tests/test_fbp_fdk.py, tests/test_vcd.py, tests/test_denoiser.py, tests/test_prox.py',
    }


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MBIRJAX_REFERENCE_ROOT')
    if not root:
        sys.exit('usage: %s <mbirjax reference root> (or set MBIRJAX_REFERENCE_ROOT)' % sys.argv[0])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'acceptance_bounds.json')
    with open(out, 'w') as f:
        json.dump(extract(root), f, indent=1)
    print('wrote', out)
