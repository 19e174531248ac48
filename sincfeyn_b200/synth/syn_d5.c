/* Synthetic Sinc-sum integrand, d = 5, splitmix64 seed 1: written by sincfeyn_b200/synth/mksynth.py */
#include "common.h"
#include "sqsynth.h"
static const double SYA_syn_d5[5]={1.3498423627584213,1.6186726358940517,1.9565041303801944,1.1665388255836582,1.166397051239537};
static const double SYB_syn_d5[5]={0.52578878382352201,0.75469737352834598,0.046134359701962779,-0.42898263120606672,0.58799321132461113};
#define REAL double
#define FN(x) x##_d
static REAL FN(f_syn_d5)(const REAL *sf, REAL *ab){
  REAL x=0, p=1, js=1;
  for(int i=0;i<5;i++){
    const REAL z=SQ_LOG(sf[i]);
    const REAL e=SQ_EXP(SYA_syn_d5[i]*z+SYB_syn_d5[i]);
    p=p*2/(e+1/e);
    x=x+SQ_EXP(-RABS(z));
    js=js*sf[i];
  }
  const REAL ex=SQ_EXP(x*1e-9);
  *ab=(ex+1)*1e9*p/js;
  return (ex-1)*1e9*p/js;
}
#undef REAL
#undef FN
#define REAL QREAL
#define FN(x) x##_q
static REAL FN(f_syn_d5)(const REAL *sf, REAL *ab){
  REAL x=0, p=1, js=1;
  for(int i=0;i<5;i++){
    const REAL z=SQ_LOG(sf[i]);
    const REAL e=SQ_EXP(SYA_syn_d5[i]*z+SYB_syn_d5[i]);
    p=p*2/(e+1/e);
    x=x+SQ_EXP(-RABS(z));
    js=js*sf[i];
  }
  const REAL ex=SQ_EXP(x*1e-9);
  *ab=(ex+1)*1e9*p/js;
  return (ex-1)*1e9*p/js;
}
#undef REAL
#undef FN
const graph_t G_syn_d5={"syn_d5","synthetic sech expm1 d=5",0,5,1,5,0,f_syn_d5_d,f_syn_d5_q,0,0};
