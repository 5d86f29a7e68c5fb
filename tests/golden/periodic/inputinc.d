ntime nrkstage istst mrestart isfera iper
3 2 2 0 0 2
cfl delt adapt relax
0.5 10.0 0. 0.
p0inf u0inf v0inf w0inf Re
0.0 10.0 0.0 0.0 0.
elliptic solver
ielast eps0 itr lord
0 1.000000e-08 100 9
itrp betap
1 0.
irl
1
dxabl dxabr dyabd dyabu dzabd dzabu
0.0 0.0 0.0 0.0 0.0 5000.0
towxl towxr towyd towyu towzd towzu
0.0 0.0 0.0 0.0 0.0 300.0
