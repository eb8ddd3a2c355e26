"""Writes the reference's CUDA source, the KERNEL string of gpu/war_gpu.py (gpu/war_gpu.py:34-260), to
oracle/_ref/war_gpu_kernel.cu unmodified, so that oracle/ref_gpu_launch.cu can compile it with nvcc for
sm_100a.  Run where the reference is mounted:  python oracle/extract_ref_kernel.py [REF_ROOT]
(REF_ROOT defaults to $WAR_REF, else the reference's mount point in the build container)."""
import ast
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WAR_REF", "/root/reference")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "war_gpu_kernel.cu")

with open(os.path.join(REF, "gpu", "war_gpu.py")) as f:
    tree = ast.parse(f.read())
src = None
for node in tree.body:
    if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "KERNEL" for t in node.targets):
        src = node.value.value
if src is None:
    raise SystemExit("KERNEL string not found")
os.makedirs(os.path.dirname(OUT), exist_ok=True)
with open(OUT, "w") as f:
    f.write(src)
print("wrote", OUT)
