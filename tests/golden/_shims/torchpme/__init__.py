"""Stand-in for torch-pme (not installed): only what the reference imports."""
