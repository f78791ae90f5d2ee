// Stand-in for FFTW's header (FFTW is absent here).  aoa-dgt's encoder header
// includes it, but every FFTW call in aoa-dgt is commented out, so nothing is
// declared.  Test infrastructure only.
#pragma once
