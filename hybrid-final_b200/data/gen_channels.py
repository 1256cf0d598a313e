"""Regenerate channels_{o2,aro2}.txt: the reaction channel list of the O2 and
Ar/O2 sets as the reference's deck reader defines it (src/start.c, the
"OxygenCase" and "Argon/OxygenCase" blocks): per channel its index, its deck
key (the JSON name of its on/off flag) and the two masses of its mofM ratio,
named as species (SP), background gas (BG) or fluid species (FG) with index.

usage: python gen_channels.py /path/to/reference/src/start.c
"""
import re
import sys

src = open(sys.argv[1]).read()
flag = re.compile(r'Coll_Flag\[(\d+)\]\.Flag\s*=\s*\(float\)json_object_get_number\(BufObject,\s*"([^"]+)"\)')
mofm = re.compile(r'Coll_Flag\[(\d+)\]\.mofM\s*=\s*(\w+)\[(\d+)\]\.mass\s*/\s*(\w+)\[(\d+)\]\.mass')


def block(start_marker, end_marker):
    a = src.index(start_marker)
    b = src.index(end_marker, a)
    return src[a:b]


def emit(text, out):
    keys = {int(m.group(1)): m.group(2) for m in flag.finditer(text)}
    ratio = {int(m.group(1)): (m.group(2), int(m.group(3)), m.group(4), int(m.group(5))) for m in mofm.finditer(text)}
    with open(out, "w") as f:
        f.write("# index key numerator denominator  (mofM = mass(numerator) / mass(denominator))\n")
        for k in sorted(keys):
            n = ratio.get(k)
            f.write(f"{k}\t{keys[k]}\t" + (f"{n[0]}{n[1]}\t{n[2]}{n[3]}" if n else "-\t-") + "\n")
    print(out, len(keys), "channels")


emit(block('"OxygenCase"', "Argon/OxygenCase"), "channels_o2.txt")
emit(block('"Argon/OxygenCase"', "Check reaction on or off"), "channels_aro2.txt")
