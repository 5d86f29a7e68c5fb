nrstart
0
ntimet
0
irestart nre
0 0
