"""Advection terms of the nonrelativistic Boltzmann equation
(bolt/src/nonrelativistic_boltzmann/advection_terms.py:28-188).

  C_q1 = v1, C_q2 = v2
  C_p  = (e/m) (E + v x B)
"""


def A_q(t, q1, q2, v1, v2, v3, params):
    return (v1, v2)


def C_q(t, q1, q2, v1, v2, v3, params):
    return (v1, v2)


def A_p(t, q1, q2, v1, v2, v3, fields_solver, params):
    return C_p(t, q1, q2, v1, v2, v3, fields_solver, params)


def C_p(t, q1, q2, v1, v2, v3, fields_solver, params):
    e = params.charge
    m = params.mass
    E1, E2, E3, B1, B2, B3 = fields_solver.get_fields()
    return ((e / m) * (E1 + v2 * B3 - v3 * B2),
            (e / m) * (E2 + v3 * B1 - v1 * B3),
            (e / m) * (E3 + v1 * B2 - v2 * B1))
