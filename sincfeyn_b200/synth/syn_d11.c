/* Synthetic Sinc-sum integrand, d = 11, splitmix64 seed 3: written by sincfeyn_b200/synth/mksynth.py */
#include "common.h"
#include "sqsynth.h"
static const double SYA_syn_d11[11]={0.67017551308573187,1.5504402703893536,1.4194620238199365,0.60930010515767807,0.82465866317222725,1.4543334735914717,0.70271878787172581,1.8330776511673164,1.2365936825921682,1.8327941024790744,1.5476542181020203};
static const double SYB_syn_d11[11]={0.42377252093931106,-0.039670991891285867,-0.32799880692035832,0.43476823642765861,0.59778051561717804,-0.38789165258611669,-0.7921891585782268,-0.65394976317828934,0.17598642358054506,0.63885031172711915,0.87140049639858952};
#define REAL double
#define FN(x) x##_d
static REAL FN(f_syn_d11)(const REAL *sf, REAL *ab){
  REAL x=0, p=1, js=1;
  for(int i=0;i<11;i++){
    const REAL z=SQ_LOG(sf[i]);
    const REAL e=SQ_EXP(SYA_syn_d11[i]*z+SYB_syn_d11[i]);
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
static REAL FN(f_syn_d11)(const REAL *sf, REAL *ab){
  REAL x=0, p=1, js=1;
  for(int i=0;i<11;i++){
    const REAL z=SQ_LOG(sf[i]);
    const REAL e=SQ_EXP(SYA_syn_d11[i]*z+SYB_syn_d11[i]);
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
const graph_t G_syn_d11={"syn_d11","synthetic sech expm1 d=11",0,11,1,11,0,f_syn_d11_d,f_syn_d11_q,0,0};
