/* Oracle shim (test infrastructure only): Corsair's crossProduct.
 * result = a x b; RHybrid calls crossProduct(B,Ue,E) to form E = -Ue x B
 * (src/particle_propagator_boris_buneman.h:105-106). */
#ifndef RHSHIM_LINEAR_ALGEBRA_H
#define RHSHIM_LINEAR_ALGEBRA_H
template<class T> inline void crossProduct(const T* a,const T* b,T* result) {
   result[0] = a[1]*b[2] - a[2]*b[1];
   result[1] = a[2]*b[0] - a[0]*b[2];
   result[2] = a[0]*b[1] - a[1]*b[0];
}
#endif
