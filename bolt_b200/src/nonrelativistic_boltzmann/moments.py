"""Velocity moments (bolt/src/nonrelativistic_boltzmann/moments.py:6-58).

Each function integrates over the p-axis (dim 0 of the AF-ordered array)."""


def integral_over_v(array, integral_measure):
    return array.sum(dim=0, keepdim=True) * integral_measure


def density(f, v1, v2, v3, integral_measure):
    return integral_over_v(f, integral_measure)


def mom_v1_bulk(f, v1, v2, v3, integral_measure):
    return integral_over_v(f * v1, integral_measure)


def mom_v2_bulk(f, v1, v2, v3, integral_measure):
    return integral_over_v(f * v2, integral_measure)


def mom_v3_bulk(f, v1, v2, v3, integral_measure):
    return integral_over_v(f * v3, integral_measure)


def energy(f, v1, v2, v3, integral_measure):
    return integral_over_v(0.5 * f * (v1 ** 2 + v2 ** 2 + v3 ** 2), integral_measure)


def energy_q1(f, v1, v2, v3, integral_measure):
    return integral_over_v(0.5 * f * v1 ** 2, integral_measure)


def energy_q2(f, v1, v2, v3, integral_measure):
    return integral_over_v(0.5 * f * v2 ** 2, integral_measure)


def energy_q3(f, v1, v2, v3, integral_measure):
    return integral_over_v(0.5 * f * v3 ** 2, integral_measure)


def q_q1(f, v1, v2, v3, integral_measure):
    return integral_over_v(f * v1 * (v1 ** 2 + v2 ** 2 + v3 ** 2), integral_measure)


def q_q2(f, v1, v2, v3, integral_measure):
    return integral_over_v(f * v2 * (v1 ** 2 + v2 ** 2 + v3 ** 2), integral_measure)


def q_q3(f, v1, v2, v3, integral_measure):
    return integral_over_v(f * v3 * (v1 ** 2 + v2 ** 2 + v3 ** 2), integral_measure)
