# test 4 inflow
test4
5   seconds
0	0
0	300
1	3600
1	14400
0	18000
