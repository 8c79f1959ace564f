; Test scan for the G-code laser path: a diagonal segment, then a straight
; one at half the feed, a jump with the beam off, and a short return pass.
G21 ; millimetres
G90
G0 X0.15 Y0.12
M3 S220
G1 X0.35 Y0.165 F60000
G1 X0.45 Y0.165 F30000
M5
G0 X0.40 Y0.10
M3 S150
G1 X0.30 Y0.10 F45000
M5
