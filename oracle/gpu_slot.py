"""Patch a copy of the reference's src/simulator.cpp so that runner_type=GPU
constructs the engine's GPU_Runner (test infrastructure: builds the
reference CLI with this engine in its GPU slot, the drop-in check).

    python3 gpu_slot.py <reference>/src/simulator.cpp <out>/simulator.cpp

Five edits, each asserted to match exactly where expected:
  1. include GPU_Runner.hpp after simulator.hpp;
  2. setENV (src/simulator.cpp:181): a GPU run opens no state files
     (state_paths is an IO-runner key);
  3. setupIni (:225-228): the GPU stub becomes `Runner = new GPU_Runner(ini)`;
  4. setupCir (:253-256): the GPU stub becomes the MEM parser
     (setupCircuit_MEM / setupSubCircuits_MEM), whose gate objects GPU_Runner
     converts;
  5. the constructor (:715): a GPU run writes no state files.
The reference sources themselves are never modified; the copy lives in the
git-ignored build directory.
"""
import sys

STUB = 'cerr << "[Config File]: GPU runner not found." << endl;\n        exit(1);'
NOT_MEM = 'env.runner_type != "MEM" && env.runner_type != "MPI_MEM"'


def patch(src: str) -> str:
    inc = '#include "simulator.hpp"\n'
    assert src.count(inc) == 1, "include line"
    src = src.replace(inc, inc + '#include "GPU_Runner.hpp"\n')
    assert src.count(NOT_MEM) == 2, "MEM runner conditions"
    src = src.replace(NOT_MEM, NOT_MEM + ' && env.runner_type != "GPU"')
    assert src.count(STUB) == 2, "GPU runner stubs"
    first = src.index(STUB)
    src = src[:first] + 'std::cout << "GPU Mode\\n";\n        Runner = new GPU_Runner(ini);' + src[first + len(STUB):]
    src = src.replace(STUB, 'if (env.is_subcircuit)\n            setupSubCircuits_MEM(cir);\n'
                            '        else\n            setupCircuit_MEM(cir);')
    assert STUB not in src
    return src


if __name__ == "__main__":
    with open(sys.argv[1]) as f:
        text = f.read()
    with open(sys.argv[2], "w") as f:
        f.write(patch(text))
