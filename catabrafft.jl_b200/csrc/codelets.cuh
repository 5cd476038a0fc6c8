// GENERATED by gen_codelets.py -- do not edit by hand.
// Straight-line DFT butterflies for radices 2, 3, 4, 5, 7, 8, 9, 16.
#pragma once
#include <type_traits>

template <typename V> struct real_of;
template <> struct real_of<double2> { typedef double R; };
template <> struct real_of<float2> { typedef float R; };
template <typename V> __device__ __forceinline__ V mk(typename real_of<V>::R x, typename real_of<V>::R y);
template <> __device__ __forceinline__ double2 mk<double2>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 mk<float2>(float x, float y) { return make_float2(x, y); }

// DFT_2, forward (w = exp(-2*pi*i/2)), in place on a[0..1]
template <typename V>
__device__ __forceinline__ void dft2(V (&a)[2]) {
    typedef typename real_of<V>::R R;
    const V a0 = a[0];
    const V a1 = a[1];
    const V t1 = mk<V>(a0.x + a1.x, a0.y + a1.y);
    const V t2 = mk<V>(a0.x - a1.x, a0.y - a1.y);
    a[0] = t1;
    a[1] = t2;
}

// DFT_3, forward (w = exp(-2*pi*i/3)), in place on a[0..2]
template <typename V>
__device__ __forceinline__ void dft3(V (&a)[3]) {
    typedef typename real_of<V>::R R;
    const V a0 = a[0];
    const V a1 = a[1];
    const V a2 = a[2];
    const V t1 = mk<V>(a1.x + a2.x, a1.y + a2.y);
    const V t2 = mk<V>(a1.x - a2.x, a1.y - a2.y);
    const V t3 = mk<V>(a0.x + t1.x, a0.y + t1.y);
    const V t4 = mk<V>(a0.x + R(-0.5) * t1.x, a0.y + R(-0.5) * t1.y);
    const V t5 = mk<V>(R(0.8660254037844386) * t2.x, R(0.8660254037844386) * t2.y);
    const V t6 = mk<V>(t4.x + t5.y, t4.y - t5.x);
    const V t7 = mk<V>(t4.x - t5.y, t4.y + t5.x);
    a[0] = t3;
    a[1] = t6;
    a[2] = t7;
}

// DFT_4, forward (w = exp(-2*pi*i/4)), in place on a[0..3]
template <typename V>
__device__ __forceinline__ void dft4(V (&a)[4]) {
    typedef typename real_of<V>::R R;
    const V a0 = a[0];
    const V a1 = a[1];
    const V a2 = a[2];
    const V a3 = a[3];
    const V t1 = mk<V>(a0.x + a2.x, a0.y + a2.y);
    const V t2 = mk<V>(a0.x - a2.x, a0.y - a2.y);
    const V t3 = mk<V>(a1.x + a3.x, a1.y + a3.y);
    const V t4 = mk<V>(a1.x - a3.x, a1.y - a3.y);
    const V t5 = mk<V>(t1.x + t3.x, t1.y + t3.y);
    const V t6 = mk<V>(t1.x - t3.x, t1.y - t3.y);
    const V t7 = mk<V>(t4.y, -t4.x);
    const V t8 = mk<V>(t2.x + t7.x, t2.y + t7.y);
    const V t9 = mk<V>(t2.x - t7.x, t2.y - t7.y);
    a[0] = t5;
    a[1] = t8;
    a[2] = t6;
    a[3] = t9;
}

// DFT_5, forward (w = exp(-2*pi*i/5)), in place on a[0..4]
template <typename V>
__device__ __forceinline__ void dft5(V (&a)[5]) {
    typedef typename real_of<V>::R R;
    const V a0 = a[0];
    const V a1 = a[1];
    const V a2 = a[2];
    const V a3 = a[3];
    const V a4 = a[4];
    const V t1 = mk<V>(a1.x + a4.x, a1.y + a4.y);
    const V t2 = mk<V>(a2.x + a3.x, a2.y + a3.y);
    const V t3 = mk<V>(a1.x - a4.x, a1.y - a4.y);
    const V t4 = mk<V>(a2.x - a3.x, a2.y - a3.y);
    const V t5 = mk<V>(a0.x + t1.x, a0.y + t1.y);
    const V t6 = mk<V>(t5.x + t2.x, t5.y + t2.y);
    const V t7 = mk<V>(a0.x + R(0.30901699437494745) * t1.x + R(-0.8090169943749475) * t2.x, a0.y + R(0.30901699437494745) * t1.y + R(-0.8090169943749475) * t2.y);
    const V t8 = mk<V>(R(0.9510565162951535) * t3.x + R(0.5877852522924731) * t4.x, R(0.9510565162951535) * t3.y + R(0.5877852522924731) * t4.y);
    const V t9 = mk<V>(t7.x + t8.y, t7.y - t8.x);
    const V t10 = mk<V>(t7.x - t8.y, t7.y + t8.x);
    const V t11 = mk<V>(a0.x + R(-0.8090169943749475) * t1.x + R(0.30901699437494745) * t2.x, a0.y + R(-0.8090169943749475) * t1.y + R(0.30901699437494745) * t2.y);
    const V t12 = mk<V>(R(0.5877852522924731) * t3.x + R(-0.9510565162951535) * t4.x, R(0.5877852522924731) * t3.y + R(-0.9510565162951535) * t4.y);
    const V t13 = mk<V>(t11.x + t12.y, t11.y - t12.x);
    const V t14 = mk<V>(t11.x - t12.y, t11.y + t12.x);
    a[0] = t6;
    a[1] = t9;
    a[2] = t13;
    a[3] = t14;
    a[4] = t10;
}

// DFT_7, forward (w = exp(-2*pi*i/7)), in place on a[0..6]
template <typename V>
__device__ __forceinline__ void dft7(V (&a)[7]) {
    typedef typename real_of<V>::R R;
    const V a0 = a[0];
    const V a1 = a[1];
    const V a2 = a[2];
    const V a3 = a[3];
    const V a4 = a[4];
    const V a5 = a[5];
    const V a6 = a[6];
    const V t1 = mk<V>(a1.x + a6.x, a1.y + a6.y);
    const V t2 = mk<V>(a2.x + a5.x, a2.y + a5.y);
    const V t3 = mk<V>(a3.x + a4.x, a3.y + a4.y);
    const V t4 = mk<V>(a1.x - a6.x, a1.y - a6.y);
    const V t5 = mk<V>(a2.x - a5.x, a2.y - a5.y);
    const V t6 = mk<V>(a3.x - a4.x, a3.y - a4.y);
    const V t7 = mk<V>(a0.x + t1.x, a0.y + t1.y);
    const V t8 = mk<V>(t7.x + t2.x, t7.y + t2.y);
    const V t9 = mk<V>(t8.x + t3.x, t8.y + t3.y);
    const V t10 = mk<V>(a0.x + R(0.6234898018587335) * t1.x + R(-0.2225209339563144) * t2.x + R(-0.9009688679024191) * t3.x, a0.y + R(0.6234898018587335) * t1.y + R(-0.2225209339563144) * t2.y + R(-0.9009688679024191) * t3.y);
    const V t11 = mk<V>(R(0.7818314824680298) * t4.x + R(0.9749279121818236) * t5.x + R(0.4338837391175581) * t6.x, R(0.7818314824680298) * t4.y + R(0.9749279121818236) * t5.y + R(0.4338837391175581) * t6.y);
    const V t12 = mk<V>(t10.x + t11.y, t10.y - t11.x);
    const V t13 = mk<V>(t10.x - t11.y, t10.y + t11.x);
    const V t14 = mk<V>(a0.x + R(-0.2225209339563144) * t1.x + R(-0.9009688679024191) * t2.x + R(0.6234898018587335) * t3.x, a0.y + R(-0.2225209339563144) * t1.y + R(-0.9009688679024191) * t2.y + R(0.6234898018587335) * t3.y);
    const V t15 = mk<V>(R(0.9749279121818236) * t4.x + R(-0.4338837391175581) * t5.x + R(-0.7818314824680298) * t6.x, R(0.9749279121818236) * t4.y + R(-0.4338837391175581) * t5.y + R(-0.7818314824680298) * t6.y);
    const V t16 = mk<V>(t14.x + t15.y, t14.y - t15.x);
    const V t17 = mk<V>(t14.x - t15.y, t14.y + t15.x);
    const V t18 = mk<V>(a0.x + R(-0.9009688679024191) * t1.x + R(0.6234898018587335) * t2.x + R(-0.2225209339563144) * t3.x, a0.y + R(-0.9009688679024191) * t1.y + R(0.6234898018587335) * t2.y + R(-0.2225209339563144) * t3.y);
    const V t19 = mk<V>(R(0.4338837391175581) * t4.x + R(-0.7818314824680298) * t5.x + R(0.9749279121818236) * t6.x, R(0.4338837391175581) * t4.y + R(-0.7818314824680298) * t5.y + R(0.9749279121818236) * t6.y);
    const V t20 = mk<V>(t18.x + t19.y, t18.y - t19.x);
    const V t21 = mk<V>(t18.x - t19.y, t18.y + t19.x);
    a[0] = t9;
    a[1] = t12;
    a[2] = t16;
    a[3] = t20;
    a[4] = t21;
    a[5] = t17;
    a[6] = t13;
}

// DFT_8, forward (w = exp(-2*pi*i/8)), in place on a[0..7]
template <typename V>
__device__ __forceinline__ void dft8(V (&a)[8]) {
    typedef typename real_of<V>::R R;
    const V a0 = a[0];
    const V a1 = a[1];
    const V a2 = a[2];
    const V a3 = a[3];
    const V a4 = a[4];
    const V a5 = a[5];
    const V a6 = a[6];
    const V a7 = a[7];
    const V t1 = mk<V>(a0.x + a4.x, a0.y + a4.y);
    const V t2 = mk<V>(a0.x - a4.x, a0.y - a4.y);
    const V t3 = mk<V>(a2.x + a6.x, a2.y + a6.y);
    const V t4 = mk<V>(a2.x - a6.x, a2.y - a6.y);
    const V t5 = mk<V>(t1.x + t3.x, t1.y + t3.y);
    const V t6 = mk<V>(t1.x - t3.x, t1.y - t3.y);
    const V t7 = mk<V>(t4.y, -t4.x);
    const V t8 = mk<V>(t2.x + t7.x, t2.y + t7.y);
    const V t9 = mk<V>(t2.x - t7.x, t2.y - t7.y);
    const V t10 = mk<V>(a1.x + a5.x, a1.y + a5.y);
    const V t11 = mk<V>(a1.x - a5.x, a1.y - a5.y);
    const V t12 = mk<V>(a3.x + a7.x, a3.y + a7.y);
    const V t13 = mk<V>(a3.x - a7.x, a3.y - a7.y);
    const V t14 = mk<V>(t10.x + t12.x, t10.y + t12.y);
    const V t15 = mk<V>(t10.x - t12.x, t10.y - t12.y);
    const V t16 = mk<V>(t13.y, -t13.x);
    const V t17 = mk<V>(t11.x + t16.x, t11.y + t16.y);
    const V t18 = mk<V>(t11.x - t16.x, t11.y - t16.y);
    const V t19 = mk<V>(t5.x + t14.x, t5.y + t14.y);
    const V t20 = mk<V>(t5.x - t14.x, t5.y - t14.y);
    const V t21 = mk<V>(R(0.7071067811865476) * (t17.x + t17.y), R(0.7071067811865476) * (t17.y - t17.x));
    const V t22 = mk<V>(t8.x + t21.x, t8.y + t21.y);
    const V t23 = mk<V>(t8.x - t21.x, t8.y - t21.y);
    const V t24 = mk<V>(t15.y, -t15.x);
    const V t25 = mk<V>(t6.x + t24.x, t6.y + t24.y);
    const V t26 = mk<V>(t6.x - t24.x, t6.y - t24.y);
    const V t27 = mk<V>(R(0.7071067811865476) * (t18.y - t18.x), -R(0.7071067811865476) * (t18.x + t18.y));
    const V t28 = mk<V>(t9.x + t27.x, t9.y + t27.y);
    const V t29 = mk<V>(t9.x - t27.x, t9.y - t27.y);
    a[0] = t19;
    a[1] = t22;
    a[2] = t25;
    a[3] = t28;
    a[4] = t20;
    a[5] = t23;
    a[6] = t26;
    a[7] = t29;
}

// DFT_9, forward (w = exp(-2*pi*i/9)), in place on a[0..8]
template <typename V>
__device__ __forceinline__ void dft9(V (&a)[9]) {
    typedef typename real_of<V>::R R;
    const V a0 = a[0];
    const V a1 = a[1];
    const V a2 = a[2];
    const V a3 = a[3];
    const V a4 = a[4];
    const V a5 = a[5];
    const V a6 = a[6];
    const V a7 = a[7];
    const V a8 = a[8];
    const V t1 = mk<V>(a3.x + a6.x, a3.y + a6.y);
    const V t2 = mk<V>(a3.x - a6.x, a3.y - a6.y);
    const V t3 = mk<V>(a0.x + t1.x, a0.y + t1.y);
    const V t4 = mk<V>(a0.x + R(-0.5) * t1.x, a0.y + R(-0.5) * t1.y);
    const V t5 = mk<V>(R(0.8660254037844386) * t2.x, R(0.8660254037844386) * t2.y);
    const V t6 = mk<V>(t4.x + t5.y, t4.y - t5.x);
    const V t7 = mk<V>(t4.x - t5.y, t4.y + t5.x);
    const V t8 = mk<V>(a4.x + a7.x, a4.y + a7.y);
    const V t9 = mk<V>(a4.x - a7.x, a4.y - a7.y);
    const V t10 = mk<V>(a1.x + t8.x, a1.y + t8.y);
    const V t11 = mk<V>(a1.x + R(-0.5) * t8.x, a1.y + R(-0.5) * t8.y);
    const V t12 = mk<V>(R(0.8660254037844386) * t9.x, R(0.8660254037844386) * t9.y);
    const V t13 = mk<V>(t11.x + t12.y, t11.y - t12.x);
    const V t14 = mk<V>(t11.x - t12.y, t11.y + t12.x);
    const V t15 = mk<V>(a5.x + a8.x, a5.y + a8.y);
    const V t16 = mk<V>(a5.x - a8.x, a5.y - a8.y);
    const V t17 = mk<V>(a2.x + t15.x, a2.y + t15.y);
    const V t18 = mk<V>(a2.x + R(-0.5) * t15.x, a2.y + R(-0.5) * t15.y);
    const V t19 = mk<V>(R(0.8660254037844386) * t16.x, R(0.8660254037844386) * t16.y);
    const V t20 = mk<V>(t18.x + t19.y, t18.y - t19.x);
    const V t21 = mk<V>(t18.x - t19.y, t18.y + t19.x);
    const V t22 = mk<V>(t10.x + t17.x, t10.y + t17.y);
    const V t23 = mk<V>(t10.x - t17.x, t10.y - t17.y);
    const V t24 = mk<V>(t3.x + t22.x, t3.y + t22.y);
    const V t25 = mk<V>(t3.x + R(-0.5) * t22.x, t3.y + R(-0.5) * t22.y);
    const V t26 = mk<V>(R(0.8660254037844386) * t23.x, R(0.8660254037844386) * t23.y);
    const V t27 = mk<V>(t25.x + t26.y, t25.y - t26.x);
    const V t28 = mk<V>(t25.x - t26.y, t25.y + t26.x);
    const V t29 = mk<V>(t13.x * R(0.766044443118978) + t13.y * R(0.6427876096865394), t13.y * R(0.766044443118978) - t13.x * R(0.6427876096865394));
    const V t30 = mk<V>(t20.x * R(0.17364817766693036) + t20.y * R(0.984807753012208), t20.y * R(0.17364817766693036) - t20.x * R(0.984807753012208));
    const V t31 = mk<V>(t29.x + t30.x, t29.y + t30.y);
    const V t32 = mk<V>(t29.x - t30.x, t29.y - t30.y);
    const V t33 = mk<V>(t6.x + t31.x, t6.y + t31.y);
    const V t34 = mk<V>(t6.x + R(-0.5) * t31.x, t6.y + R(-0.5) * t31.y);
    const V t35 = mk<V>(R(0.8660254037844386) * t32.x, R(0.8660254037844386) * t32.y);
    const V t36 = mk<V>(t34.x + t35.y, t34.y - t35.x);
    const V t37 = mk<V>(t34.x - t35.y, t34.y + t35.x);
    const V t38 = mk<V>(t14.x * R(0.17364817766693036) + t14.y * R(0.984807753012208), t14.y * R(0.17364817766693036) - t14.x * R(0.984807753012208));
    const V t39 = mk<V>(t21.x * R(-0.9396926207859084) + t21.y * R(0.3420201433256687), t21.y * R(-0.9396926207859084) - t21.x * R(0.3420201433256687));
    const V t40 = mk<V>(t38.x + t39.x, t38.y + t39.y);
    const V t41 = mk<V>(t38.x - t39.x, t38.y - t39.y);
    const V t42 = mk<V>(t7.x + t40.x, t7.y + t40.y);
    const V t43 = mk<V>(t7.x + R(-0.5) * t40.x, t7.y + R(-0.5) * t40.y);
    const V t44 = mk<V>(R(0.8660254037844386) * t41.x, R(0.8660254037844386) * t41.y);
    const V t45 = mk<V>(t43.x + t44.y, t43.y - t44.x);
    const V t46 = mk<V>(t43.x - t44.y, t43.y + t44.x);
    a[0] = t24;
    a[1] = t33;
    a[2] = t42;
    a[3] = t27;
    a[4] = t36;
    a[5] = t45;
    a[6] = t28;
    a[7] = t37;
    a[8] = t46;
}

// DFT_16, forward (w = exp(-2*pi*i/16)), in place on a[0..15]
template <typename V>
__device__ __forceinline__ void dft16(V (&a)[16]) {
    typedef typename real_of<V>::R R;
    const V a0 = a[0];
    const V a1 = a[1];
    const V a2 = a[2];
    const V a3 = a[3];
    const V a4 = a[4];
    const V a5 = a[5];
    const V a6 = a[6];
    const V a7 = a[7];
    const V a8 = a[8];
    const V a9 = a[9];
    const V a10 = a[10];
    const V a11 = a[11];
    const V a12 = a[12];
    const V a13 = a[13];
    const V a14 = a[14];
    const V a15 = a[15];
    const V t1 = mk<V>(a0.x + a8.x, a0.y + a8.y);
    const V t2 = mk<V>(a0.x - a8.x, a0.y - a8.y);
    const V t3 = mk<V>(a4.x + a12.x, a4.y + a12.y);
    const V t4 = mk<V>(a4.x - a12.x, a4.y - a12.y);
    const V t5 = mk<V>(t1.x + t3.x, t1.y + t3.y);
    const V t6 = mk<V>(t1.x - t3.x, t1.y - t3.y);
    const V t7 = mk<V>(t4.y, -t4.x);
    const V t8 = mk<V>(t2.x + t7.x, t2.y + t7.y);
    const V t9 = mk<V>(t2.x - t7.x, t2.y - t7.y);
    const V t10 = mk<V>(a2.x + a10.x, a2.y + a10.y);
    const V t11 = mk<V>(a2.x - a10.x, a2.y - a10.y);
    const V t12 = mk<V>(a6.x + a14.x, a6.y + a14.y);
    const V t13 = mk<V>(a6.x - a14.x, a6.y - a14.y);
    const V t14 = mk<V>(t10.x + t12.x, t10.y + t12.y);
    const V t15 = mk<V>(t10.x - t12.x, t10.y - t12.y);
    const V t16 = mk<V>(t13.y, -t13.x);
    const V t17 = mk<V>(t11.x + t16.x, t11.y + t16.y);
    const V t18 = mk<V>(t11.x - t16.x, t11.y - t16.y);
    const V t19 = mk<V>(t5.x + t14.x, t5.y + t14.y);
    const V t20 = mk<V>(t5.x - t14.x, t5.y - t14.y);
    const V t21 = mk<V>(R(0.7071067811865476) * (t17.x + t17.y), R(0.7071067811865476) * (t17.y - t17.x));
    const V t22 = mk<V>(t8.x + t21.x, t8.y + t21.y);
    const V t23 = mk<V>(t8.x - t21.x, t8.y - t21.y);
    const V t24 = mk<V>(t15.y, -t15.x);
    const V t25 = mk<V>(t6.x + t24.x, t6.y + t24.y);
    const V t26 = mk<V>(t6.x - t24.x, t6.y - t24.y);
    const V t27 = mk<V>(R(0.7071067811865476) * (t18.y - t18.x), -R(0.7071067811865476) * (t18.x + t18.y));
    const V t28 = mk<V>(t9.x + t27.x, t9.y + t27.y);
    const V t29 = mk<V>(t9.x - t27.x, t9.y - t27.y);
    const V t30 = mk<V>(a1.x + a9.x, a1.y + a9.y);
    const V t31 = mk<V>(a1.x - a9.x, a1.y - a9.y);
    const V t32 = mk<V>(a5.x + a13.x, a5.y + a13.y);
    const V t33 = mk<V>(a5.x - a13.x, a5.y - a13.y);
    const V t34 = mk<V>(t30.x + t32.x, t30.y + t32.y);
    const V t35 = mk<V>(t30.x - t32.x, t30.y - t32.y);
    const V t36 = mk<V>(t33.y, -t33.x);
    const V t37 = mk<V>(t31.x + t36.x, t31.y + t36.y);
    const V t38 = mk<V>(t31.x - t36.x, t31.y - t36.y);
    const V t39 = mk<V>(a3.x + a11.x, a3.y + a11.y);
    const V t40 = mk<V>(a3.x - a11.x, a3.y - a11.y);
    const V t41 = mk<V>(a7.x + a15.x, a7.y + a15.y);
    const V t42 = mk<V>(a7.x - a15.x, a7.y - a15.y);
    const V t43 = mk<V>(t39.x + t41.x, t39.y + t41.y);
    const V t44 = mk<V>(t39.x - t41.x, t39.y - t41.y);
    const V t45 = mk<V>(t42.y, -t42.x);
    const V t46 = mk<V>(t40.x + t45.x, t40.y + t45.y);
    const V t47 = mk<V>(t40.x - t45.x, t40.y - t45.y);
    const V t48 = mk<V>(t34.x + t43.x, t34.y + t43.y);
    const V t49 = mk<V>(t34.x - t43.x, t34.y - t43.y);
    const V t50 = mk<V>(R(0.7071067811865476) * (t46.x + t46.y), R(0.7071067811865476) * (t46.y - t46.x));
    const V t51 = mk<V>(t37.x + t50.x, t37.y + t50.y);
    const V t52 = mk<V>(t37.x - t50.x, t37.y - t50.y);
    const V t53 = mk<V>(t44.y, -t44.x);
    const V t54 = mk<V>(t35.x + t53.x, t35.y + t53.y);
    const V t55 = mk<V>(t35.x - t53.x, t35.y - t53.y);
    const V t56 = mk<V>(R(0.7071067811865476) * (t47.y - t47.x), -R(0.7071067811865476) * (t47.x + t47.y));
    const V t57 = mk<V>(t38.x + t56.x, t38.y + t56.y);
    const V t58 = mk<V>(t38.x - t56.x, t38.y - t56.y);
    const V t59 = mk<V>(t19.x + t48.x, t19.y + t48.y);
    const V t60 = mk<V>(t19.x - t48.x, t19.y - t48.y);
    const V t61 = mk<V>(t51.x * R(0.9238795325112867) + t51.y * R(0.3826834323650898), t51.y * R(0.9238795325112867) - t51.x * R(0.3826834323650898));
    const V t62 = mk<V>(t22.x + t61.x, t22.y + t61.y);
    const V t63 = mk<V>(t22.x - t61.x, t22.y - t61.y);
    const V t64 = mk<V>(R(0.7071067811865476) * (t54.x + t54.y), R(0.7071067811865476) * (t54.y - t54.x));
    const V t65 = mk<V>(t25.x + t64.x, t25.y + t64.y);
    const V t66 = mk<V>(t25.x - t64.x, t25.y - t64.y);
    const V t67 = mk<V>(t57.x * R(0.3826834323650898) + t57.y * R(0.9238795325112867), t57.y * R(0.3826834323650898) - t57.x * R(0.9238795325112867));
    const V t68 = mk<V>(t28.x + t67.x, t28.y + t67.y);
    const V t69 = mk<V>(t28.x - t67.x, t28.y - t67.y);
    const V t70 = mk<V>(t49.y, -t49.x);
    const V t71 = mk<V>(t20.x + t70.x, t20.y + t70.y);
    const V t72 = mk<V>(t20.x - t70.x, t20.y - t70.y);
    const V t73 = mk<V>(t52.x * R(-0.3826834323650898) + t52.y * R(0.9238795325112867), t52.y * R(-0.3826834323650898) - t52.x * R(0.9238795325112867));
    const V t74 = mk<V>(t23.x + t73.x, t23.y + t73.y);
    const V t75 = mk<V>(t23.x - t73.x, t23.y - t73.y);
    const V t76 = mk<V>(R(0.7071067811865476) * (t55.y - t55.x), -R(0.7071067811865476) * (t55.x + t55.y));
    const V t77 = mk<V>(t26.x + t76.x, t26.y + t76.y);
    const V t78 = mk<V>(t26.x - t76.x, t26.y - t76.y);
    const V t79 = mk<V>(t58.x * R(-0.9238795325112867) + t58.y * R(0.3826834323650898), t58.y * R(-0.9238795325112867) - t58.x * R(0.3826834323650898));
    const V t80 = mk<V>(t29.x + t79.x, t29.y + t79.y);
    const V t81 = mk<V>(t29.x - t79.x, t29.y - t79.y);
    a[0] = t59;
    a[1] = t62;
    a[2] = t65;
    a[3] = t68;
    a[4] = t71;
    a[5] = t74;
    a[6] = t77;
    a[7] = t80;
    a[8] = t60;
    a[9] = t63;
    a[10] = t66;
    a[11] = t69;
    a[12] = t72;
    a[13] = t75;
    a[14] = t78;
    a[15] = t81;
}

template <int RADIX, typename V> __device__ __forceinline__ void dft(V (&a)[RADIX]) {
    if constexpr (RADIX == 2) dft2(a);
    else if constexpr (RADIX == 3) dft3(a);
    else if constexpr (RADIX == 4) dft4(a);
    else if constexpr (RADIX == 5) dft5(a);
    else if constexpr (RADIX == 7) dft7(a);
    else if constexpr (RADIX == 8) dft8(a);
    else if constexpr (RADIX == 9) dft9(a);
    else if constexpr (RADIX == 16) dft16(a);
}
