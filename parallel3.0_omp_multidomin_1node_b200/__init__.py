"""Package root: the importable package is ``tdbem`` in this directory."""
