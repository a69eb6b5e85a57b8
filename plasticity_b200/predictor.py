"""Learned per-node Newton predictor (placeholder until trained weights exist)."""


def weights_available() -> bool:
    return False


def load_into(model) -> None:
    raise RuntimeError("no trained predictor weights")
