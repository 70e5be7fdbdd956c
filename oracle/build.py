"""Build the oracle (test infrastructure): gcc -O2 oracle.c -> oracle/_build/liboracle.so."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build():
    out = os.path.join(HERE, "_build")
    os.makedirs(out, exist_ok=True)
    lib = os.path.join(out, "liboracle.so")
    src = os.path.join(HERE, "oracle.c")
    if os.path.exists(lib) and os.path.getmtime(lib) >= os.path.getmtime(src):
        return lib
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-o", lib, src, "-lm"], check=True)
    return lib


if __name__ == "__main__":
    print(build())
