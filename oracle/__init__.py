"""TEST INFRASTRUCTURE ONLY: the CPU oracle for the AN operator path.

See oracle/oracle.py.  Nothing in the ahead_b200 package imports this.
"""
