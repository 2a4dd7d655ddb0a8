// common.cuh -- shared definitions for the B200 CW-FDTD library.
//
// Scalar steady-state fit (the 2-sample and 3-sample amplitude/phase formulas)
// and the ramped source envelope are written once here as __host__ __device__
// functions: the exported scalar ABI entry points (FDTD_calc_phase_3T, ...)
// and the device probe/extraction kernels evaluate the same code.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define FDTD_HD __host__ __device__ __forceinline__

namespace fdtdb {

struct c128 { double real, imag; };

// ---------------------------------------------------------------- fit math
// f(t) = A sin(t + phi) sampled at two times, no offset (src/fdtd.cpp:1445-1463).
FDTD_HD double phase_2t(double t0, double t1, double f0, double f1) {
    if (f0 == 0.0 && f1 == 0.0) return 0.0;
    return atan((f1 * sin(t0) - f0 * sin(t1)) / (f0 * cos(t1) - f1 * cos(t0)));
}

FDTD_HD double amplitude_2t(double t0, double t1, double f0, double f1, double phase) {
    if (f0 * f0 > f1 * f1) return f1 / (sin(t1) * cos(phase) + cos(t1) * sin(phase));
    return f0 / (sin(t0) * cos(phase) + cos(t0) * sin(phase));
}

// f(t) = A sin(t + phi) + B sampled at three times (src/fdtd.cpp:1465-1493).
FDTD_HD double phase_3t(double t0, double t1, double t2, double f0, double f1, double f2) {
    double f10 = f1 - f0, f21 = f2 - f1;
    if (f10 == 0.0 && f21 == 0.0) return 0.0;
    return atan2(f10 * (sin(t2) - sin(t1)) - f21 * (sin(t1) - sin(t0)),
                 f21 * (cos(t1) - cos(t0)) - f10 * (cos(t2) - cos(t1)));
}

FDTD_HD double amplitude_3t(double t0, double t1, double t2, double f0, double f1, double f2,
                            double phase) {
    double f21 = f2 - f1, f10 = f1 - f0;
    if (f21 == 0.0 && f10 == 0.0) return 0.0;
    if (f21 * f21 >= f10 * f10)
        return f21 / (cos(phase) * (sin(t2) - sin(t1)) + sin(phase) * (cos(t2) - cos(t1)));
    return f10 / (cos(phase) * (sin(t1) - sin(t0)) + sin(phase) * (cos(t1) - cos(t0)));
}

// Sine/cosine of the three sample times, evaluated once per extraction call.
struct Fit3 {
    double s0, s1, s2, c0, c1, c2;
};

FDTD_HD Fit3 make_fit3(double t0, double t1, double t2) {
    Fit3 f;
    f.s0 = sin(t0); f.s1 = sin(t1); f.s2 = sin(t2);
    f.c0 = cos(t0); f.c1 = cos(t1); f.c2 = cos(t2);
    return f;
}

// Complex phasor A e^{-i phi} of the 3-sample fit.  Folding a negative A into
// phi + pi leaves A e^{-i phi} unchanged, so with cos(phi) = X/r and
// sin(phi) = Y/r (phi = atan2(Y, X)) the phasor is f (X - iY) / (X ds + Y dc),
// where (f, ds, dc) is the reference's branch: the later difference f21 when
// f21^2 >= f10^2, otherwise f10.  The degenerate X = Y = 0 case falls back to
// the trigonometric form.
FDTD_HD c128 phasor_3t(const Fit3& F, double f0, double f1, double f2) {
    double f10 = f1 - f0, f21 = f2 - f1;
    c128 out;
    if (f10 == 0.0 && f21 == 0.0) { out.real = 0.0; out.imag = -0.0; return out; }
    double Y = f10 * (F.s2 - F.s1) - f21 * (F.s1 - F.s0);
    double X = f21 * (F.c1 - F.c0) - f10 * (F.c2 - F.c1);
    double f, ds, dc;
    if (f21 * f21 >= f10 * f10) { f = f21; ds = F.s2 - F.s1; dc = F.c2 - F.c1; }
    else { f = f10; ds = F.s1 - F.s0; dc = F.c1 - F.c0; }
    if (X == 0.0 && Y == 0.0) {
        double phi = atan2(Y, X);
        double A = f / (cos(phi) * ds + sin(phi) * dc);
        if (A < 0) { A = -A; phi += M_PI; }
        out.real = A * cos(phi);
        out.imag = -A * sin(phi);
        return out;
    }
    double g = f / (X * ds + Y * dc);
    out.real = g * X;
    out.imag = -(g * Y);
    return out;
}

// Two-sample phasor with the reference's trigonometric sequence.
FDTD_HD c128 phasor_2t(double t0, double t1, double f0, double f1) {
    double phi = phase_2t(t0, t1, f0, f1);
    double A = amplitude_2t(t0, t1, f0, f1, phi);
    if (A < 0) { A *= -1; phi += M_PI; }
    c128 out;
    out.real = A * cos(phi);
    out.imag = -A * sin(phi);
    return out;
}

// Ramped CW envelope (src/fdtd.cpp:1595-1602): the source is
// sin(t + phase) * env(t) with env = (1+m) exp(-(t-T)^2/k) - m for t <= T.
FDTD_HD double src_envelope(double t, double T, double m, double k) {
    if (t <= T) return (1 + m) * exp(-(t - T) * (t - T) / k) - m;
    return 1.0;
}

FDTD_HD double src_value(double t, double phase, double T, double m, double k) {
    if (t <= T) return sin(t + phase) * ((1 + m) * exp(-(t - T) * (t - T) / k) - m);
    return sin(t + phase);
}

}  // namespace fdtdb
