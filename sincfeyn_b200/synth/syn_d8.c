/* Synthetic Sinc-sum integrand, d = 8, splitmix64 seed 2: written by sincfeyn_b200/synth/mksynth.py */
#include "common.h"
#include "sqsynth.h"
static const double SYA_syn_d8[8]={1.3867846012971192,1.6237245258107369,1.393457122100008,1.6481287312925441,0.96738303077167109,1.0199334056175484,1.5895304217751216,1.6086309865213686};
static const double SYB_syn_d8[8]={-0.49937525561739604,0.45523192916778021,-0.32103674443953256,-0.12434760611771201,0.1115828405048731,-0.25239323884162035,0.864002126823183,-0.59321803966513054};
#define REAL double
#define FN(x) x##_d
static REAL FN(f_syn_d8)(const REAL *sf, REAL *ab){
  REAL x=0, p=1, js=1;
  for(int i=0;i<8;i++){
    const REAL z=SQ_LOG(sf[i]);
    const REAL e=SQ_EXP(SYA_syn_d8[i]*z+SYB_syn_d8[i]);
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
static REAL FN(f_syn_d8)(const REAL *sf, REAL *ab){
  REAL x=0, p=1, js=1;
  for(int i=0;i<8;i++){
    const REAL z=SQ_LOG(sf[i]);
    const REAL e=SQ_EXP(SYA_syn_d8[i]*z+SYB_syn_d8[i]);
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
const graph_t G_syn_d8={"syn_d8","synthetic sech expm1 d=8",0,8,1,8,0,f_syn_d8_d,f_syn_d8_q,0,0};
