"""Extract the reference's qGGMRF golden vectors into ``qggmrf_golden.json``.

The reference test ``tests/test_qggmrf.py`` (``test_gradient_and_hessian``, lines 81-134) holds a fixed
3x3x3 volume, fixed (p, q, T, sigma_x) and the gradient / Hessian a verified version of the reference
produced for them.  This script reads that file as text (it is never imported or executed), pulls the
literal arrays and scalars out of the function body with ``ast``, and writes them as a fixture so that the
tests can run where the reference tree is absent.

Usage: python tests/golden/make_qggmrf_golden.py <path/to/reference/root>  (or MBIRJAX_REFERENCE_ROOT=<root>)
"""
import ast
import json
import os
import sys


def _literal(node):
    # np.array([[...]], dtype=...) or a parenthesised np.array(...) -> nested list
    if isinstance(node, ast.Call):
        return ast.literal_eval(node.args[0])
    return ast.literal_eval(node)


def extract(reference_root):
    path = os.path.join(reference_root, 'tests', 'test_qggmrf.py')
    tree = ast.parse(open(path).read())
    func = next(n for n in ast.walk(tree) if isinstance(n, ast.FunctionDef) and n.name == 'test_gradient_and_hessian')
    wanted = {'grad_ref', 'hess_ref', 'p', 'q', 'T', 'sigma_x', 'flat_recon', 'recon_shape'}
    out = {}
    for stmt in func.body:
        if isinstance(stmt, ast.Assign) and len(stmt.targets) == 1 and isinstance(stmt.targets[0], ast.Name):
            name = stmt.targets[0].id
            if name in wanted and name not in out:
                out[name] = _literal(stmt.value)
    missing = wanted - set(out)
    if missing:
        raise RuntimeError('could not find %s in %s' % (sorted(missing), path))
    out['b'] = 'normalised (1,1,1,1,1,1)'
    out['source'] = 'reference tests/test_qggmrf.py:81-134 (test_gradient_and_hessian)'
    return out


if __name__ == '__main__':
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MBIRJAX_REFERENCE_ROOT')
    if not root:
        sys.exit('usage: %s <mbirjax reference root> (or set MBIRJAX_REFERENCE_ROOT)' % sys.argv[0])
    data = extract(root)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'qggmrf_golden.json')
    with open(dst, 'w') as f:
        json.dump(data, f, indent=1)
    print('wrote', dst)
