"""Recipe: compile the reference's CUDA-C plasma kernel source
(src/3+1D-UPPE-ERK4(3)IP-envelope/media_physics.py:11-67) as host C++ into
oracle/_ref/ (test infrastructure).  The source string is read out of the
reference file; nothing is copied into this repository.

The reference tree is the first command-line argument, else the environment
variable UPPE_REFERENCE, else the development container's checkout."""
import ast
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, '_ref')
MEDIA_REL = os.path.join('src', '3+1D-UPPE-ERK4(3)IP-envelope', 'media_physics.py')


def reference_root(argv=None):
    argv = sys.argv if argv is None else argv
    if __name__ == '__main__' and len(argv) > 1:
        return argv[1]
    return os.environ.get('UPPE_REFERENCE', '/root/reference')


def media_path(root=None):
    return os.path.join(root or reference_root(), MEDIA_REL)

PRELUDE = r'''
#include <math.h>
struct _uppe_dim3 { unsigned x, y, z; };
static _uppe_dim3 blockDim, blockIdx, threadIdx;
#define __global__
'''

LAUNCHER = r'''
extern "C" void _launch_plasma_integration_kernel(unsigned grid, unsigned block,
    const float* W_ion, const float* W_ava, double* rho, double* gen,
    float rate_rec, float dt, float rho_nt, int Nt, int nsp) {
  blockDim.x = block; blockDim.y = blockDim.z = 1;
  for (unsigned b = 0; b < grid; ++b) {
    blockIdx.x = b;
    for (unsigned t = 0; t < block; ++t) {
      threadIdx.x = t;
      plasma_integration_kernel(W_ion, W_ava, rho, gen, rate_rec, dt, rho_nt, Nt, nsp);
    }
  }
}
'''


def kernel_source(path=None):
    tree = ast.parse(open(path or media_path(), encoding='utf-8').read())
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(getattr(t, 'id', '') == 'PLASMA_KERNEL_CODE'
                                                for t in node.targets):
            return node.value.value
    raise RuntimeError('PLASMA_KERNEL_CODE not found')


def build(code=None):
    """Compile and return the path of the host .so (cached by source hash)."""
    if code is None:
        code = kernel_source()
    os.makedirs(OUT, exist_ok=True)
    src = PRELUDE + code + LAUNCHER
    tag = hashlib.sha1(src.encode()).hexdigest()[:12]
    cpp = os.path.join(OUT, f'plasma_kernel_{tag}.cpp')
    so = os.path.join(OUT, f'plasma_kernel_{tag}.so')
    if not os.path.exists(so):
        with open(cpp, 'w') as f:
            f.write(src)
        subprocess.check_call(['g++', '-O2', '-fPIC', '-shared', '-o', so, cpp])
    return so


if __name__ == '__main__':
    print(build())
