: A passive leak written for the runtime-registration tests: i = g (v - e) per unit area.
NEURON {
    SUFFIX userleak
    NONSPECIFIC_CURRENT i
    RANGE g, e
}

UNITS {
    (mA) = (milliamp)
    (mV) = (millivolt)
    (S) = (siemens)
}

PARAMETER {
    g = 0.001 (S/cm2) <0,1e9>
    e = -70 (mV)
}

ASSIGNED {
    v (mV)
    i (mA/cm2)
}

BREAKPOINT {
    i = g*(v - e)
}
