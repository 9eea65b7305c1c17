"""Makes the scene fixtures that the CPU side of the benchmark reads (test infrastructure, like the rest of oracle/).

shell_large.npz: the 20 m gridshell (20 m hexagonal plan, 60 laths per family at 0.33 m, 3.8 cm segments, supports
lifted 0-2 m by a seeded field; 81,180 nodes, 81,000 segments, 8,190 crossings), built once by the package's scene
builder and saved as a model.  The benchmark's reference arm relaxes it with the oracle alone, so that arm's process
never loads the CUDA library; tests/test_scene.py checks that the fixture is still what the scene builder makes.

    python oracle/scenes/make_scenes.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    sys.path.insert(0, ROOT)
    import weavesim_b200 as ws
    md = ws.configs.shell_large()
    path = os.path.join(HERE, "shell_large.npz")
    md.save(path)
    print(f"{path}: n {md.n}, m {md.m}, K {md.K}, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
