"""TEST INFRASTRUCTURE ONLY — the reference's hard-coded INPUT values (DP/buildInput.cu:10-69)
as a case struct built without the product library, for the oracle's own runs (bench.py's
reference arm).  Field names follow the reference's struct INPUT (DP/strdata.h:49-98); the
extension fields keep their zero (reference-behaviour) values."""
from __future__ import annotations


def reference_defaults():
    from fooskagpu_b200._lib import FgCase   # the struct layout only; no library is loaded
    c = FgCase()
    vals = dict(dt=0.0, adaptDt=1, adaptDtItr=100, maxDt=1e-8, cfl=0.1, avfMin=1e-4, rkSteps=1, finalTime=3.5e-3,
                exportTime=2.0e-5, restartStep=100000, restartFlag=0, neglectX=0, neglectY=0, neglectZ=0,
                nMaterials=2, NEQ=10, scale=0.001, viscFlag=1, turbulence=1, woodsFlag=1, thermFntRlxFlag=0,
                thermRlxRate=0.5, thermUrf=0.8, thermItrMax=25, chemFlag=1, chemFntRlxFlag=0, chemRlxRate=0.0,
                chemUrf=0.5, chemItrMax=40, chemCondesation=0, chemLimit=20e-4, consCalcFlag=1, consCalcIvar=9,
                satTempUrf=0.8)
    for k, v in vals.items():
        setattr(c, k, v)
    phase = dict(gamma=(2.17290, 1.4588), pInf=(114907765.0, 0.0), Cp=(1854.4, 965.98),
                 eta=(-302568.5557, 9741.04362), satConst=(-488.9933492, 297.63826), dynVisc=(1.8e-4, 1.99e-5))
    for k, (a, b) in phase.items():
        getattr(c, k)[0] = a
        getattr(c, k)[1] = b
    return c
