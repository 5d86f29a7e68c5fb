mg_flag
0
smoothing
sm_flag1 sm_flag2
1 0
omega
1.0
sweeps
itrp1 itrp2 itrp_c1 itrp_c2 itrp_cc
1 0 0 0 0
match_flag
1
