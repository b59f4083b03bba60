"""Contraction forms that tests pin when they compare a single context with
the batch path bit for bit: the batch path runs the carried-temporal-line
forms (10 mixed, 7 FP64), a context the temporal-gauge form by default."""


def carried_form(prec: str) -> int:
    return 7 if prec == "fp64" else 10
