"""opt_einsum stand-in whose path search declines, so the reference falls
back to its plain ``tf.einsum`` branch (same contraction, summation order
aside)."""


def contract_path(*args, **kwargs):
    raise NotImplementedError("path search not provided")


def contract(*args, **kwargs):
    raise NotImplementedError("contract not provided")


def get_symbol(i):
    return "abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ"[i]
