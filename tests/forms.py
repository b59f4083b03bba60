"""The carried-temporal-line contraction form a context runs when the
temporal-gauge form is switched off (10 mixed, 7 FP64; also the form of
lattices smeared without projection); tests pin it to compare the
carried-line shapes with each other, or the two forms with each other."""


def carried_form(prec: str) -> int:
    return 7 if prec == "fp64" else 10
