"""Compiles the C host programs of tests/c_abi against include/mdff_gpu.h and
the in-tree libmdff_gpu.so (gcc; used by the tests)."""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def compile_c(name, out_dir):
    """Path of the built executable for tests/c_abi/<name>.c, or None without gcc."""
    gcc = shutil.which("gcc")
    if gcc is None:
        return None
    libdir = os.path.join(ROOT, "mdff_b200")
    exe = os.path.join(str(out_dir), name)
    subprocess.run([gcc, "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, name + ".c"), "-L", libdir, "-lmdff_gpu",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    return exe
