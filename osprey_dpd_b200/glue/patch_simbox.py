"""Writes the OSPREY_DPD_CUDA copy of the reference's SimBox.cpp: the file as
it is, plus the include of osprey_dpd_glue.h and, first in the body of
CSimBox::Evolve (SimBox.cpp:977-1120), the call that hands the step to the
engine.  Nothing else changes.

    python patch_simbox.py <reference SimBox.cpp> <output SimBox.cpp>
"""
import re
import sys

INCLUDE = '\n#if OSPREY_DPD_CUDA\n#include "osprey_dpd_glue.h"\n#endif\n'

HOOK = """
#if OSPREY_DPD_CUDA
	// The step runs on the B200 engine; on steps where beads are read the
	// engine's state is written back (per-bead stress here: CSimBox is a
	// friend of CAbstractBead).
	{
		OspreyDpdSync ospreySync = {0, 0};
		const bool ospreyRead = TimeToSample() || TimeToDisplay() || TimeToRestart() || m_SimTime == m_TotalTime;
		const bool ospreyRenorm = IsRenormalisationOn() && m_SimTime % m_RenormalisationPeriod == 0;
		if (OspreyDpdEvolve(this, m_SimTime, ospreyRead, ospreyRenorm, &ospreySync))
		{
			if (ospreySync.stress9)
				for (size_t k = 0; k < ospreySync.beads->size(); ++k)
					for (int q = 0; q < 9; ++q)
						(*ospreySync.beads)[k]->m_Stress[q] = ospreySync.stress9[9 * k + q];
			return;
		}
	}
#endif
"""


def patch(src: str) -> str:
    inc = re.search(r'^#include\s+"SimBox\.h"\s*$', src, flags=re.M)   # unconditional, near the top
    if not inc:
        raise SystemExit("patch_simbox: #include \"SimBox.h\" not found")
    at = inc.end()
    src = src[:at] + INCLUDE + src[at:]
    m = re.search(r'^void CSimBox::Evolve\(\)\s*\n\{', src, flags=re.M)
    if not m:
        raise SystemExit("patch_simbox: CSimBox::Evolve not found")
    return src[:m.end()] + HOOK + src[m.end():]


def main():
    src = open(sys.argv[1], encoding="latin-1").read()
    with open(sys.argv[2], "w", encoding="latin-1") as fh:
        fh.write(patch(src))


if __name__ == "__main__":
    main()
