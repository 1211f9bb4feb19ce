"""Command-line drop-ins for the SIE-GSTC applications, on the sieb200 C ABI."""
