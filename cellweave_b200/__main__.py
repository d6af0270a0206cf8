"""``python -m cellweave_b200 run.toml [--steps N] [--histories H] [--out DIR]``:
a configuration file's run on the device (cellweave_b200.config.main)."""
from .config import main

main()
