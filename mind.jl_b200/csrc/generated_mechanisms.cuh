/*
 * generated_mechanisms.cuh -- CUDA C emitted from MOD files by mind_b200.nmodl.  Do not edit:
 * regenerate with mind.jl_b200/csrc/gen_mechanisms.py.  Each mechanism's kind code is
 * MIND_MECH_GENERATED + its index below; its fields are its columns in order.
 */
#pragma once

#include "gen_runtime.cuh"

namespace mind {
namespace gen {

/* SEClamp (point mechanism), generated from SEClamp.mod by
 * mind_b200.nmodl.  Columns: 0 rs, 1 dur1, 2 amp1, 3 dur2, 4 amp2, 5 dur3, 6 amp3, 7 i, 8 vc, 9 tc2, 10 tc3, 11 on. */
struct M0_SEClamp {
    static constexpr int kColumns = 12;
    struct S {
        double rs;
        double dur1;
        double amp1;
        double dur2;
        double amp2;
        double dur3;
        double amp3;
        double i;
        double vc;
        double tc2;
        double tc3;
        double on;
        double v, t, dt, celsius;
    };
    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {
        s.rs = r.at(0);
        s.dur1 = r.at(1);
        s.amp1 = r.at(2);
        s.dur2 = r.at(3);
        s.amp2 = r.at(4);
        s.dur3 = r.at(5);
        s.amp3 = r.at(6);
        s.i = r.at(7);
        s.vc = r.at(8);
        s.tc2 = r.at(9);
        s.tc3 = r.at(10);
        s.on = r.at(11);
        s.v = r.v;
        s.t = r.t;
        s.dt = r.dt;
        s.celsius = r.celsius;
    }
    __device__ static __forceinline__ void p_icur(S &s) {
        if ((s.on != 0.0)) {
            s.i = ((s.vc - s.v) / s.rs);
        } else {
            s.i = 0.0;
        }
    }
    __device__ static __forceinline__ void p_vstim(S &s) {
        s.on = 1.0;
        if ((s.dur1 != 0.0)) {
        }
        if ((s.dur2 != 0.0)) {
        }
        if ((s.dur3 != 0.0)) {
        }
        if ((s.t < s.dur1)) {
            s.vc = s.amp1;
        } else {
            if ((s.t < s.tc2)) {
                s.vc = s.amp2;
            } else {
                if ((s.t < s.tc3)) {
                    s.vc = s.amp3;
                } else {
                    s.vc = 0.0;
                    s.on = 0.0;
                }
            }
        }
        p_icur(s);
    }
    __device__ static __forceinline__ void initial(const MindGenRow &r) {
        S s;
        load(s, r);
        s.tc2 = (s.dur1 + s.dur2);
        s.tc3 = (s.tc2 + s.dur3);
        s.on = 0.0;
        r.at(9) = s.tc2;
        r.at(10) = s.tc3;
        r.at(11) = s.on;
    }
    __device__ static __forceinline__ double current(const MindGenRow &r) {
        S s;
        load(s, r);
        p_vstim(s);
        r.at(7) = s.i;
        r.at(8) = s.vc;
        r.at(11) = s.on;
        double value = 0.0;
        value -= s.i;
        return value;
    }
    __device__ static __forceinline__ void advance(const MindGenRow &r) {
        S s;
        load(s, r);
        p_icur(s);
        r.at(7) = s.i;
    }
};

/* VClamp (point mechanism), generated from VClamp.mod by
 * mind_b200.nmodl.  Columns: 0 dur[0], 1 dur[1], 2 dur[2], 3 amp[0], 4 amp[1], 5 amp[2], 6 gain, 7 rstim, 8 tau1, 9 tau2, 10 e0, 11 vo0, 12 vi0, 13 fac, 14 e, 15 vo, 16 vi, 17 i, 18 stim, 19 tc. */
struct M1_VClamp {
    static constexpr int kColumns = 20;
    struct S {
        double dur[3];
        double amp[3];
        double gain;
        double rstim;
        double tau1;
        double tau2;
        double e0;
        double vo0;
        double vi0;
        double fac;
        double e;
        double vo;
        double vi;
        double i;
        double stim;
        double tc;
        double v, t, dt, celsius;
    };
    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {
        s.dur[0] = r.at(0);
        s.dur[1] = r.at(1);
        s.dur[2] = r.at(2);
        s.amp[0] = r.at(3);
        s.amp[1] = r.at(4);
        s.amp[2] = r.at(5);
        s.gain = r.at(6);
        s.rstim = r.at(7);
        s.tau1 = r.at(8);
        s.tau2 = r.at(9);
        s.e0 = r.at(10);
        s.vo0 = r.at(11);
        s.vi0 = r.at(12);
        s.fac = r.at(13);
        s.e = r.at(14);
        s.vo = r.at(15);
        s.vi = r.at(16);
        s.i = r.at(17);
        s.stim = r.at(18);
        s.tc = r.at(19);
        s.v = r.v;
        s.t = r.t;
        s.dt = r.dt;
        s.celsius = r.celsius;
    }
    __device__ static __forceinline__ void p_vstim(S &s) {
        double l_j = 0.0;
        double l_selected = 0.0;
        s.tc = 0.0;
        l_j = 0.0;
        l_selected = 0.0;
        for (int guard_ = 0; guard_ < (1 << 20) && ((l_j < 3.0) && (!(l_selected != 0.0))); ++guard_) {
            s.stim = s.amp[mind_gen_index(l_j, 3)];
            s.tc = (s.tc + s.dur[mind_gen_index(l_j, 3)]);
            if ((s.t < s.tc)) {
                s.tc = (s.tc + 100.0);
                l_selected = 1.0;
            }
            l_j = (l_j + 1.0);
        }
    }
    __device__ static __forceinline__ void p_clamp(S &s) {
        double l_t1 = 0.0;
        double l_t2 = 0.0;
        l_t1 = (s.tau1 / s.dt);
        l_t2 = (s.tau2 / s.dt);
        s.e = (((((1.0 + l_t1) * (((1.0 - s.fac) * s.v) + (((s.fac * l_t2) * s.vo0) / (1.0 + l_t2)))) - s.stim) - (l_t1 * (s.vi0 - s.e0))) / ((2.0 + l_t1) + ((((1.0 + l_t1) * s.fac) * s.gain) / (1.0 + l_t2))));
        s.vo = (((l_t2 * s.vo0) - (s.gain * s.e)) / (1.0 + l_t2));
        s.vi = ((s.v + (s.fac * s.vo)) - (s.fac * s.v));
    }
    __device__ static __forceinline__ double f_icur(S &s) {
        double ret_ = 0.0;
        if ((s.t > s.tc)) {
            s.e0 = 0.0;
            s.vo0 = 0.0;
            ret_ = 0.0;
        } else {
            p_clamp(s);
            ret_ = ((s.vo - s.v) / s.rstim);
        }
        return ret_;
    }
    __device__ static __forceinline__ void p_update(S &s) {
        s.i = f_icur(s);
        s.e0 = s.e;
        s.vo0 = s.vo;
        s.vi0 = s.vi;
    }
    __device__ static __forceinline__ void initial(const MindGenRow &r) {
        S s;
        load(s, r);
        s.e0 = 0.0;
        s.vo = s.v;
        s.vo0 = s.v;
        s.vi = s.v;
        s.vi0 = s.v;
        s.e = 0.0;
        r.at(10) = s.e0;
        r.at(11) = s.vo0;
        r.at(12) = s.vi0;
        r.at(14) = s.e;
        r.at(15) = s.vo;
        r.at(16) = s.vi;
    }
    __device__ static __forceinline__ double current(const MindGenRow &r) {
        S s;
        load(s, r);
        p_vstim(s);
        s.i = f_icur(s);
        r.at(10) = s.e0;
        r.at(11) = s.vo0;
        r.at(14) = s.e;
        r.at(15) = s.vo;
        r.at(16) = s.vi;
        r.at(17) = s.i;
        r.at(18) = s.stim;
        r.at(19) = s.tc;
        double value = 0.0;
        value -= s.i;
        return value;
    }
    __device__ static __forceinline__ void advance(const MindGenRow &r) {
        S s;
        load(s, r);
        p_update(s);
        r.at(10) = s.e0;
        r.at(11) = s.vo0;
        r.at(12) = s.vi0;
        r.at(14) = s.e;
        r.at(15) = s.vo;
        r.at(16) = s.vi;
        r.at(17) = s.i;
    }
};

/* hh (density mechanism), generated from hh.mod by
 * mind_b200.nmodl.  Columns: 0 gnabar, 1 gkbar, 2 gl, 3 el, 4 m, 5 h, 6 n, 7 ena, 8 ek, 9 gna, 10 gk, 11 ina, 12 ik, 13 il, 14 minf, 15 hinf, 16 ninf, 17 mtau, 18 htau, 19 ntau. */
struct M2_hh {
    static constexpr int kColumns = 20;
    struct S {
        double gnabar;
        double gkbar;
        double gl;
        double el;
        double m;
        double h;
        double n;
        double ena;
        double ek;
        double gna;
        double gk;
        double ina;
        double ik;
        double il;
        double minf;
        double hinf;
        double ninf;
        double mtau;
        double htau;
        double ntau;
        double v, t, dt, celsius;
    };
    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {
        s.gnabar = r.at(0);
        s.gkbar = r.at(1);
        s.gl = r.at(2);
        s.el = r.at(3);
        s.m = r.at(4);
        s.h = r.at(5);
        s.n = r.at(6);
        s.ena = r.at(7);
        s.ek = r.at(8);
        s.gna = r.at(9);
        s.gk = r.at(10);
        s.ina = r.at(11);
        s.ik = r.at(12);
        s.il = r.at(13);
        s.minf = r.at(14);
        s.hinf = r.at(15);
        s.ninf = r.at(16);
        s.mtau = r.at(17);
        s.htau = r.at(18);
        s.ntau = r.at(19);
        s.v = r.v;
        s.t = r.t;
        s.dt = r.dt;
        s.celsius = r.celsius;
    }
    __device__ static __forceinline__ void p_rates(S &s, double a_v) {
        double l_alpha = 0.0;
        double l_beta = 0.0;
        double l_sum = 0.0;
        double l_q10 = 0.0;
        l_q10 = mind_pow(3.0, ((s.celsius - 6.3) / 10.0));
        l_alpha = (0.1 * f_vtrap(s, (-(a_v + 40.0)), 10.0));
        l_beta = (4.0 * mind_exp(((-(a_v + 65.0)) / 18.0)));
        l_sum = (l_alpha + l_beta);
        s.mtau = (1.0 / (l_q10 * l_sum));
        s.minf = (l_alpha / l_sum);
        l_alpha = (0.07 * mind_exp(((-(a_v + 65.0)) / 20.0)));
        l_beta = (1.0 / (mind_exp(((-(a_v + 35.0)) / 10.0)) + 1.0));
        l_sum = (l_alpha + l_beta);
        s.htau = (1.0 / (l_q10 * l_sum));
        s.hinf = (l_alpha / l_sum);
        l_alpha = (0.01 * f_vtrap(s, (-(a_v + 55.0)), 10.0));
        l_beta = (0.125 * mind_exp(((-(a_v + 65.0)) / 80.0)));
        l_sum = (l_alpha + l_beta);
        s.ntau = (1.0 / (l_q10 * l_sum));
        s.ninf = (l_alpha / l_sum);
    }
    __device__ static __forceinline__ double f_vtrap(S &s, double a_x, double a_y) {
        double ret_ = 0.0;
        if ((fabs((a_x / a_y)) < 1e-06)) {
            ret_ = (a_y * (1.0 - ((a_x / a_y) / 2.0)));
        } else {
            ret_ = (a_x / (mind_exp((a_x / a_y)) - 1.0));
        }
        return ret_;
    }
    __device__ static __forceinline__ void d_states(S &s) {
        p_rates(s, s.v);
        s.m = s.m + (1.0 - mind_exp(s.dt * (-1.0 / s.mtau))) * (s.minf - s.m);
        s.h = s.h + (1.0 - mind_exp(s.dt * (-1.0 / s.htau))) * (s.hinf - s.h);
        s.n = s.n + (1.0 - mind_exp(s.dt * (-1.0 / s.ntau))) * (s.ninf - s.n);
    }
    __device__ static __forceinline__ void initial(const MindGenRow &r) {
        S s;
        load(s, r);
        p_rates(s, s.v);
        s.m = s.minf;
        s.h = s.hinf;
        s.n = s.ninf;
        r.at(4) = s.m;
        r.at(5) = s.h;
        r.at(6) = s.n;
        r.at(14) = s.minf;
        r.at(15) = s.hinf;
        r.at(16) = s.ninf;
        r.at(17) = s.mtau;
        r.at(18) = s.htau;
        r.at(19) = s.ntau;
    }
    __device__ static __forceinline__ double current(const MindGenRow &r) {
        S s;
        load(s, r);
        s.gna = ((((s.gnabar * s.m) * s.m) * s.m) * s.h);
        s.ina = (s.gna * (s.v - s.ena));
        s.gk = ((((s.gkbar * s.n) * s.n) * s.n) * s.n);
        s.ik = (s.gk * (s.v - s.ek));
        s.il = (s.gl * (s.v - s.el));
        r.at(9) = s.gna;
        r.at(10) = s.gk;
        r.at(11) = s.ina;
        r.at(12) = s.ik;
        r.at(13) = s.il;
        double value = 0.0;
        value += s.il;
        value += s.ina;
        value += s.ik;
        return value;
    }
    __device__ static __forceinline__ void advance(const MindGenRow &r) {
        S s;
        load(s, r);
        d_states(s);
        r.at(4) = s.m;
        r.at(5) = s.h;
        r.at(6) = s.n;
        r.at(14) = s.minf;
        r.at(15) = s.hinf;
        r.at(16) = s.ninf;
        r.at(17) = s.mtau;
        r.at(18) = s.htau;
        r.at(19) = s.ntau;
    }
};

/* pas (density mechanism), generated from pas.mod by
 * mind_b200.nmodl.  Columns: 0 g, 1 e, 2 i. */
struct M3_pas {
    static constexpr int kColumns = 3;
    struct S {
        double g;
        double e;
        double i;
        double v, t, dt, celsius;
    };
    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {
        s.g = r.at(0);
        s.e = r.at(1);
        s.i = r.at(2);
        s.v = r.v;
        s.t = r.t;
        s.dt = r.dt;
        s.celsius = r.celsius;
    }
    __device__ static __forceinline__ void initial(const MindGenRow &r) {
        S s;
        load(s, r);
    }
    __device__ static __forceinline__ double current(const MindGenRow &r) {
        S s;
        load(s, r);
        s.i = (s.g * (s.v - s.e));
        r.at(2) = s.i;
        double value = 0.0;
        value += s.i;
        return value;
    }
    __device__ static __forceinline__ void advance(const MindGenRow &r) {
        S s;
        load(s, r);
    }
};

/* ExpSyn (point mechanism), generated from ExpSyn.mod by
 * mind_b200.nmodl.  Columns: 0 tau, 1 e, 2 g, 3 i. */
struct M4_ExpSyn {
    static constexpr int kColumns = 4;
    struct S {
        double tau;
        double e;
        double g;
        double i;
        double v, t, dt, celsius;
    };
    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {
        s.tau = r.at(0);
        s.e = r.at(1);
        s.g = r.at(2);
        s.i = r.at(3);
        s.v = r.v;
        s.t = r.t;
        s.dt = r.dt;
        s.celsius = r.celsius;
    }
    __device__ static __forceinline__ void d_state(S &s) {
        s.g = s.g + (1.0 - mind_exp(s.dt * (-1.0 / s.tau))) * (0.0 - s.g);
    }
    __device__ static __forceinline__ void initial(const MindGenRow &r) {
        S s;
        load(s, r);
        s.g = 0.0;
        r.at(2) = s.g;
    }
    __device__ static __forceinline__ double current(const MindGenRow &r) {
        S s;
        load(s, r);
        s.i = (s.g * (s.v - s.e));
        r.at(3) = s.i;
        double value = 0.0;
        value += s.i;
        return value;
    }
    __device__ static __forceinline__ void advance(const MindGenRow &r) {
        S s;
        load(s, r);
        d_state(s);
        r.at(2) = s.g;
    }
    __device__ static __forceinline__ void receive(const MindGenRow &r, double w_, double flag_) {
        S s;
        load(s, r);
        s.g = (s.g + w_);
        r.at(2) = s.g;
    }
};

/* Exp2Syn (point mechanism), generated from Exp2Syn.mod by
 * mind_b200.nmodl.  Columns: 0 tau1, 1 tau2, 2 e, 3 A, 4 B, 5 i, 6 g, 7 factor. */
struct M5_Exp2Syn {
    static constexpr int kColumns = 8;
    struct S {
        double tau1;
        double tau2;
        double e;
        double A;
        double B;
        double i;
        double g;
        double factor;
        double v, t, dt, celsius;
    };
    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {
        s.tau1 = r.at(0);
        s.tau2 = r.at(1);
        s.e = r.at(2);
        s.A = r.at(3);
        s.B = r.at(4);
        s.i = r.at(5);
        s.g = r.at(6);
        s.factor = r.at(7);
        s.v = r.v;
        s.t = r.t;
        s.dt = r.dt;
        s.celsius = r.celsius;
    }
    __device__ static __forceinline__ void d_state(S &s) {
        s.A = s.A + (1.0 - mind_exp(s.dt * (-1.0 / s.tau1))) * (0.0 - s.A);
        s.B = s.B + (1.0 - mind_exp(s.dt * (-1.0 / s.tau2))) * (0.0 - s.B);
    }
    __device__ static __forceinline__ void initial(const MindGenRow &r) {
        S s;
        load(s, r);
        double l_tp = 0.0;
        if (((s.tau1 / s.tau2) > 0.9999)) {
            s.tau1 = (0.9999 * s.tau2);
        }
        if (((s.tau1 / s.tau2) < 1e-09)) {
            s.tau1 = (s.tau2 * 1e-09);
        }
        s.A = 0.0;
        s.B = 0.0;
        l_tp = (((s.tau1 * s.tau2) / (s.tau2 - s.tau1)) * mind_log((s.tau2 / s.tau1)));
        s.factor = ((-mind_exp(((-l_tp) / s.tau1))) + mind_exp(((-l_tp) / s.tau2)));
        s.factor = (1.0 / s.factor);
        r.at(0) = s.tau1;
        r.at(3) = s.A;
        r.at(4) = s.B;
        r.at(7) = s.factor;
    }
    __device__ static __forceinline__ double current(const MindGenRow &r) {
        S s;
        load(s, r);
        s.g = (s.B - s.A);
        s.i = (s.g * (s.v - s.e));
        r.at(5) = s.i;
        r.at(6) = s.g;
        double value = 0.0;
        value += s.i;
        return value;
    }
    __device__ static __forceinline__ void advance(const MindGenRow &r) {
        S s;
        load(s, r);
        d_state(s);
        r.at(3) = s.A;
        r.at(4) = s.B;
    }
    __device__ static __forceinline__ void receive(const MindGenRow &r, double w_, double flag_) {
        S s;
        load(s, r);
        s.A = (s.A + (w_ * s.factor));
        s.B = (s.B + (w_ * s.factor));
        r.at(3) = s.A;
        r.at(4) = s.B;
    }
};

/* IClamp (point mechanism), generated from IClamp.mod by
 * mind_b200.nmodl.  Columns: 0 del, 1 dur, 2 amp, 3 i. */
struct M6_IClamp {
    static constexpr int kColumns = 4;
    struct S {
        double del;
        double dur;
        double amp;
        double i;
        double v, t, dt, celsius;
    };
    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {
        s.del = r.at(0);
        s.dur = r.at(1);
        s.amp = r.at(2);
        s.i = r.at(3);
        s.v = r.v;
        s.t = r.t;
        s.dt = r.dt;
        s.celsius = r.celsius;
    }
    __device__ static __forceinline__ void initial(const MindGenRow &r) {
        S s;
        load(s, r);
        s.i = 0.0;
        r.at(3) = s.i;
    }
    __device__ static __forceinline__ double current(const MindGenRow &r) {
        S s;
        load(s, r);
        if (((s.t < (s.del + s.dur)) && (s.t >= s.del))) {
            s.i = s.amp;
        } else {
            s.i = 0.0;
        }
        r.at(3) = s.i;
        double value = 0.0;
        value -= s.i;
        return value;
    }
    __device__ static __forceinline__ void advance(const MindGenRow &r) {
        S s;
        load(s, r);
    }
};

/* AlphaSynapse (point mechanism), generated from AlphaSynapse.mod by
 * mind_b200.nmodl.  Columns: 0 onset, 1 tau, 2 gmax, 3 e, 4 i, 5 g. */
struct M7_AlphaSynapse {
    static constexpr int kColumns = 6;
    struct S {
        double onset;
        double tau;
        double gmax;
        double e;
        double i;
        double g;
        double v, t, dt, celsius;
    };
    __device__ static __forceinline__ void load(S &s, const MindGenRow &r) {
        s.onset = r.at(0);
        s.tau = r.at(1);
        s.gmax = r.at(2);
        s.e = r.at(3);
        s.i = r.at(4);
        s.g = r.at(5);
        s.v = r.v;
        s.t = r.t;
        s.dt = r.dt;
        s.celsius = r.celsius;
    }
    __device__ static __forceinline__ double f_alpha(S &s, double a_x) {
        double ret_ = 0.0;
        if (((a_x < 0.0) || (a_x > 10.0))) {
            ret_ = 0.0;
        } else {
            ret_ = (a_x * mind_exp((1.0 - a_x)));
        }
        return ret_;
    }
    __device__ static __forceinline__ void initial(const MindGenRow &r) {
        S s;
        load(s, r);
    }
    __device__ static __forceinline__ double current(const MindGenRow &r) {
        S s;
        load(s, r);
        if ((s.gmax != 0.0)) {
        }
        s.g = (s.gmax * f_alpha(s, ((s.t - s.onset) / s.tau)));
        s.i = (s.g * (s.v - s.e));
        r.at(4) = s.i;
        r.at(5) = s.g;
        double value = 0.0;
        value += s.i;
        return value;
    }
    __device__ static __forceinline__ void advance(const MindGenRow &r) {
        S s;
        load(s, r);
    }
};

}  // namespace gen

constexpr int kGeneratedCount = 8;
struct GenMechanism {
    const char *name;
    int32_t point;          // 1: POINT_PROCESS, 0: density (SUFFIX)
    int32_t net_receive;    // NET_RECEIVE arity (0: none)
    int32_t first_field;    // into kGenFieldNames / kGenDefaults
    int32_t n_fields;
    uint64_t digest;        // first 16 hex digits of the MOD source's SHA-256
    const char *ion_reads;  // "field ion ..." pairs a USEION READ fills from the ion species
};
static const char *const kGenFieldNames[] = {"rs", "dur1", "amp1", "dur2", "amp2", "dur3", "amp3", "i", "vc", "tc2", "tc3", "on", "dur[0]", "dur[1]", "dur[2]", "amp[0]", "amp[1]", "amp[2]", "gain", "rstim", "tau1", "tau2", "e0", "vo0", "vi0", "fac", "e", "vo", "vi", "i", "stim", "tc", "gnabar", "gkbar", "gl", "el", "m", "h", "n", "ena", "ek", "gna", "gk", "ina", "ik", "il", "minf", "hinf", "ninf", "mtau", "htau", "ntau", "g", "e", "i", "tau", "e", "g", "i", "tau1", "tau2", "e", "A", "B", "i", "g", "factor", "del", "dur", "amp", "i", "onset", "tau", "gmax", "e", "i", "g"};
static const double kGenDefaults[] = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 100000.0, 1.0, 0.001, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.12, 0.036, 0.0003, -54.3, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.001, -70.0, 0.0, 0.1, 0.0, 0.0, 0.0, 0.1, 10.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.1, 0.0, 0.0, 0.0, 0.0};
static const GenMechanism kGenMechanisms[] = {
    {"SEClamp", 1, 0, 0, 12, 0xBDD7FEA652CA1EBAull, ""},
    {"VClamp", 1, 0, 12, 20, 0xB82001FEA2C4B6DAull, ""},
    {"hh", 0, 0, 32, 20, 0x06A1D0784470B30Bull, "ena na ek k"},
    {"pas", 0, 0, 52, 3, 0x7C96D2C7CB7FE0C5ull, ""},
    {"ExpSyn", 1, 1, 55, 4, 0x9704333E132D681Cull, ""},
    {"Exp2Syn", 1, 1, 59, 8, 0xC42E524B775C6D4Dull, ""},
    {"IClamp", 1, 0, 67, 4, 0x6EB0551A76C267F8ull, ""},
    {"AlphaSynapse", 1, 0, 71, 6, 0x29B06B38B5009424ull, ""},
};

#ifdef MIND_GEN_BUILTIN_DISPATCH
__device__ __forceinline__ void gen_builtin_initial(int32_t id, const MindGenRow &r) {
    switch (id) {
        case 0: gen::M0_SEClamp::initial(r); return;
        case 1: gen::M1_VClamp::initial(r); return;
        case 2: gen::M2_hh::initial(r); return;
        case 3: gen::M3_pas::initial(r); return;
        case 4: gen::M4_ExpSyn::initial(r); return;
        case 5: gen::M5_Exp2Syn::initial(r); return;
        case 6: gen::M6_IClamp::initial(r); return;
        case 7: gen::M7_AlphaSynapse::initial(r); return;
        default: break;
    }
}
__device__ __forceinline__ double gen_builtin_current(int32_t id, const MindGenRow &r) {
    switch (id) {
        case 0: return gen::M0_SEClamp::current(r);
        case 1: return gen::M1_VClamp::current(r);
        case 2: return gen::M2_hh::current(r);
        case 3: return gen::M3_pas::current(r);
        case 4: return gen::M4_ExpSyn::current(r);
        case 5: return gen::M5_Exp2Syn::current(r);
        case 6: return gen::M6_IClamp::current(r);
        case 7: return gen::M7_AlphaSynapse::current(r);
        default: break;
    }
    return 0.0;
}
__device__ __forceinline__ void gen_builtin_advance(int32_t id, const MindGenRow &r) {
    switch (id) {
        case 0: gen::M0_SEClamp::advance(r); return;
        case 1: gen::M1_VClamp::advance(r); return;
        case 2: gen::M2_hh::advance(r); return;
        case 3: gen::M3_pas::advance(r); return;
        case 4: gen::M4_ExpSyn::advance(r); return;
        case 5: gen::M5_Exp2Syn::advance(r); return;
        case 6: gen::M6_IClamp::advance(r); return;
        case 7: gen::M7_AlphaSynapse::advance(r); return;
        default: break;
    }
}
__device__ __forceinline__ void gen_builtin_receive(int32_t id, const MindGenRow &r, double w, double flag) {
    switch (id) {
        case 4: gen::M4_ExpSyn::receive(r, w, flag); return;
        case 5: gen::M5_Exp2Syn::receive(r, w, flag); return;
        default: break;
    }
}
#else
__device__ __forceinline__ void gen_initial(int32_t id, const MindGenRow &r) {
    switch (id) {
        case 0: gen::M0_SEClamp::initial(r); return;
        case 1: gen::M1_VClamp::initial(r); return;
        case 2: gen::M2_hh::initial(r); return;
        case 3: gen::M3_pas::initial(r); return;
        case 4: gen::M4_ExpSyn::initial(r); return;
        case 5: gen::M5_Exp2Syn::initial(r); return;
        case 6: gen::M6_IClamp::initial(r); return;
        case 7: gen::M7_AlphaSynapse::initial(r); return;
        default: break;
    }
}
__device__ __forceinline__ double gen_current(int32_t id, const MindGenRow &r) {
    switch (id) {
        case 0: return gen::M0_SEClamp::current(r);
        case 1: return gen::M1_VClamp::current(r);
        case 2: return gen::M2_hh::current(r);
        case 3: return gen::M3_pas::current(r);
        case 4: return gen::M4_ExpSyn::current(r);
        case 5: return gen::M5_Exp2Syn::current(r);
        case 6: return gen::M6_IClamp::current(r);
        case 7: return gen::M7_AlphaSynapse::current(r);
        default: break;
    }
    return 0.0;
}
__device__ __forceinline__ void gen_advance(int32_t id, const MindGenRow &r) {
    switch (id) {
        case 0: gen::M0_SEClamp::advance(r); return;
        case 1: gen::M1_VClamp::advance(r); return;
        case 2: gen::M2_hh::advance(r); return;
        case 3: gen::M3_pas::advance(r); return;
        case 4: gen::M4_ExpSyn::advance(r); return;
        case 5: gen::M5_Exp2Syn::advance(r); return;
        case 6: gen::M6_IClamp::advance(r); return;
        case 7: gen::M7_AlphaSynapse::advance(r); return;
        default: break;
    }
}
__device__ __forceinline__ void gen_receive(int32_t id, const MindGenRow &r, double w, double flag) {
    switch (id) {
        case 4: gen::M4_ExpSyn::receive(r, w, flag); return;
        case 5: gen::M5_Exp2Syn::receive(r, w, flag); return;
        default: break;
    }
}
#endif

}  // namespace mind
